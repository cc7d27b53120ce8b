// xorwow_jump.h -- jump a XORWOW state ahead by 2^32 (or 2^67) draws.
//
// The reference seeds every frame of every pixel with
// curand_init(seed, pixel, frame * 2^32) (core/random.cuh:31-39), so frame f+1
// of a pixel starts exactly 2^32 draws after frame f.  This file advances a
// state by that distance without curand's general skip-ahead.
//
// Method: the generator is Marsaglia's xorwow ("Xorshift RNGs", J. Stat. Softw.
// 8(14), 2003): a 160-bit xorshift register (x, y, z, w, v) updated by
//     t = x ^ (x >> 2); x = y; y = z; z = w; w = v; v = (v ^ (v << 4)) ^ (t ^ (t << 1))
// plus a Weyl counter d += 362437 that is added to the output.  The register
// update is linear over GF(2), so n steps are the 160x160 bit matrix A^n
// (jump-ahead for F2-linear generators, Haramoto et al., INFORMS J. Comput.
// 2008).  A^(2^32) is built on the host by 32 squarings of A, and applied as 40
// lookups of 4-bit chunks (T[c][nibble] = A^(2^32) * (nibble << 4c), 12.8 KB).
// The counter moves by 362437 * 2^32 = 0 (mod 2^32), so d is unchanged.
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

namespace ar {

constexpr int kJumpChunks = 40;                    // 160 bits / 4
constexpr int kJumpWords = kJumpChunks * 5 * 16;   // table words, layout [chunk][word][nibble]

struct Bits160 { uint32_t w[5]; };

inline Bits160 xorwow_register_step(const Bits160& s)
{
    Bits160 r;
    const uint32_t t = s.w[0] ^ (s.w[0] >> 2);
    r.w[0] = s.w[1];
    r.w[1] = s.w[2];
    r.w[2] = s.w[3];
    r.w[3] = s.w[4];
    r.w[4] = (s.w[4] ^ (s.w[4] << 4)) ^ (t ^ (t << 1));
    return r;
}

// Column-major GF(2) matrix: col[i] = M * e_i.
struct Mat160 { Bits160 col[160]; };

inline Bits160 mat_apply(const Mat160& m, const Bits160& v)
{
    Bits160 r = {{0, 0, 0, 0, 0}};
    for (int i = 0; i < 160; ++i)
        if ((v.w[i >> 5] >> (i & 31)) & 1u)
            for (int k = 0; k < 5; ++k) r.w[k] ^= m.col[i].w[k];
    return r;
}

// Table of A^(2^p) for the device apply (layout [chunk][word][nibble]).
inline std::vector<uint32_t> xorwow_jump_table_pow2(int p)
{
    Mat160 m;
    for (int i = 0; i < 160; ++i) {
        Bits160 e = {{0, 0, 0, 0, 0}};
        e.w[i >> 5] = 1u << (i & 31);
        m.col[i] = xorwow_register_step(e);
    }
    for (int sq = 0; sq < p; ++sq) {  // A^(2^(k+1)) = A^(2^k) * A^(2^k)
        Mat160 n;
        for (int i = 0; i < 160; ++i) n.col[i] = mat_apply(m, m.col[i]);
        m = n;
    }
    std::vector<uint32_t> t(kJumpWords, 0u);
    for (int c = 0; c < kJumpChunks; ++c)
        for (int nib = 0; nib < 16; ++nib) {
            Bits160 acc = {{0, 0, 0, 0, 0}};
            for (int b = 0; b < 4; ++b)
                if ((nib >> b) & 1)
                    for (int k = 0; k < 5; ++k) acc.w[k] ^= m.col[4 * c + b].w[k];
            for (int k = 0; k < 5; ++k) t[(c * 5 + k) * 16 + nib] = acc.w[k];
        }
    return t;
}

// Host apply of a table built by xorwow_jump_table_pow2.
inline Bits160 xorwow_jump_apply(const std::vector<uint32_t>& table, const Bits160& v)
{
    Bits160 r = {{0, 0, 0, 0, 0}};
    for (int c = 0; c < kJumpChunks; ++c) {
        const uint32_t nib = (v.w[c >> 3] >> (4 * (c & 7))) & 15u;
        for (int k = 0; k < 5; ++k) r.w[k] ^= table[(c * 5 + k) * 16 + nib];
    }
    return r;
}

// The frame jump: 2^32 draws.
inline std::vector<uint32_t> xorwow_jump_table_2p32() { return xorwow_jump_table_pow2(32); }

#ifdef __CUDACC__
// v (the five register words, curand order v[0..4]) <- M v for the jump M of
// a table built by xorwow_jump_table_pow2 (A^(2^32): one frame; A^(2^67): one
// curand subsequence), with the table staged in shared memory.
__device__ __forceinline__ void xorwow_jump(uint32_t v[5], const uint32_t* __restrict__ table)
{
    uint32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0, r4 = 0;
#pragma unroll
    for (int c = 0; c < kJumpChunks; ++c) {
        const uint32_t nib = (v[c >> 3] >> (4 * (c & 7))) & 15u;
        const uint32_t* row = table + c * 80 + nib;
        r0 ^= row[0];
        r1 ^= row[16];
        r2 ^= row[32];
        r3 ^= row[48];
        r4 ^= row[64];
    }
    v[0] = r0; v[1] = r1; v[2] = r2; v[3] = r3; v[4] = r4;
}
#endif

}  // namespace ar
