// Host check of the XORWOW frame jump (csrc/xorwow_jump.h), run by
// tests/test_cpu_host_logic.py.  Prints "OK" and exits 0 when
//   (1) the table of A^(2^16) equals 65536 explicit register steps, and
//   (2) the table of A^(2^32) equals 65536 applications of the A^(2^16) table,
//   (3) the tables of A^(2^33) and of A^(2^67) (one curand subsequence, the
//       per-pixel initialisation's jump) equal two applications of the tables
//       of A^(2^32) and A^(2^66),
// for a handful of register states; exits 1 on the first mismatch.
#include <cstdio>

#include "../../aperturerendererv3-optix-geometry_b200/csrc/xorwow_jump.h"

using ar::Bits160;

static bool same(const Bits160& a, const Bits160& b)
{
    for (int k = 0; k < 5; ++k)
        if (a.w[k] != b.w[k]) return false;
    return true;
}

int main()
{
    const std::vector<uint32_t> t16 = ar::xorwow_jump_table_pow2(16);
    const std::vector<uint32_t> t32 = ar::xorwow_jump_table_2p32();
    const std::vector<uint32_t> t33 = ar::xorwow_jump_table_pow2(33);
    const std::vector<uint32_t> t66 = ar::xorwow_jump_table_pow2(66);
    const std::vector<uint32_t> t67 = ar::xorwow_jump_table_pow2(67);
    const Bits160 states[] = {
        {{0x12345678u, 0x9abcdef0u, 0x0badf00du, 0xdeadbeefu, 0x13579bdfu}},
        {{1u, 0u, 0u, 0u, 0u}},
        {{0u, 0u, 0u, 0u, 0x80000000u}},
        {{0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu}},
    };
    for (const Bits160& s : states) {
        Bits160 x = s;
        for (int i = 0; i < 65536; ++i) x = ar::xorwow_register_step(x);
        if (!same(x, ar::xorwow_jump_apply(t16, s))) { std::printf("MISMATCH 2^16\n"); return 1; }
        Bits160 y = s;
        for (int i = 0; i < 65536; ++i) y = ar::xorwow_jump_apply(t16, y);
        if (!same(y, ar::xorwow_jump_apply(t32, s))) { std::printf("MISMATCH 2^32\n"); return 1; }
        if (!same(ar::xorwow_jump_apply(t32, ar::xorwow_jump_apply(t32, s)), ar::xorwow_jump_apply(t33, s))) {
            std::printf("MISMATCH 2^33\n");
            return 1;
        }
        if (!same(ar::xorwow_jump_apply(t66, ar::xorwow_jump_apply(t66, s)), ar::xorwow_jump_apply(t67, s))) {
            std::printf("MISMATCH 2^67\n");
            return 1;
        }
    }
    std::printf("OK\n");
    return 0;
}
