// shading.cuh -- BSDF sampling and evaluation, light sampling and sky of the
// reference's RGB path loop, as device functions of the shade kernels.
//
// Each function restates the reference function named beside it with the same
// expression order (see detmath.h for the rounding contract).
#pragma once

#include <curand_kernel.h>

#include "traverse.cuh"

namespace ar {

// Per-path random stream: curand XORWOW, Rand1 (core/random.cuh:41-44).
struct Rng {
    curandStateXORWOW_t st;
    int used;
    __device__ __forceinline__ float next()
    {
        ++used;
        return curand_uniform(&st);  // Rand1 (random.cuh:41-44)
    }
};

__device__ __forceinline__ f3 xyz(float4 a) { return mk(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(f3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// INTERSECT_EPS(d) for d = 0..8 (config.cuh:3), computed on the host with the
// fixed exp of detmath.h and uploaded once per device (set_intersect_eps).
__constant__ float c_eps_tab[9];

// ------------------------------------------------------------------ shading helpers
// Shading inputs of a hit.  In spectral mode albedo and emissive hold the
// colour's response at the path's wavelength in all three components, ior and
// sigma_a their values at that wavelength, and `spectral` selects the scalar
// forms of the few expressions that mix channels (GGX lobe probability).
struct GB {
    f3 albedo, emissive;
    float specular, metallic, roughness, ior, sigma_a;
    float abbe, tilt;
    bool spectral;
};

__device__ __forceinline__ GB load_gb(const MaterialRec& m)
{
    GB g;
    g.albedo = mk(m.albedo[0], m.albedo[1], m.albedo[2]);
    g.emissive = mk(m.emissive[0], m.emissive[1], m.emissive[2]);
    g.specular = m.specular; g.metallic = m.metallic; g.roughness = m.roughness; g.ior = m.ior; g.sigma_a = m.sigma_a;
    g.abbe = m.abbe; g.tilt = m.tilt;
    g.spectral = false;
    return g;
}

// GGX lobe-selection probability: clamp(luminance(F0)) in RGB, clamp(F0) at one
// wavelength (material.cuh:283-289, 372-378).
__device__ __forceinline__ float ggx_pspec(const GB& g, f3 F0)
{
    return clampf(g.spectral ? F0.x : luminance(F0), 0.1f, 0.9f);
}

// BuildTangentBasis / BuildTangentBasisRandom (vector.cuh:264-283)
__device__ __forceinline__ void tangent_basis(f3 n, f3& t, f3& b)
{
    const f3 a = (fabsf(n.z) < 0.999f) ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    t = normalize(cross(a, n));
    b = cross(n, t);
}
__device__ __forceinline__ void tangent_basis_random(f3 n, f3& t, f3& b, float e)
{
    const f3 a = (fabsf(n.z) < 0.999f) ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    const f3 t0 = normalize(cross(a, n));
    const f3 b0 = cross(n, t0);
    float sn, cs;
    sincos_det(e * kPi * 2.0f, &sn, &cs);
    t = t0 * cs + b0 * sn;
    b = t0 * (-sn) + b0 * cs;
}
// SampleCosineWeightedHemisphere + ConcentricSampleDisk (sample.cuh:63-108)
__device__ __forceinline__ f3 sample_cosine(float e0, float e1, float e2, f3 n, float& pdf)
{
    f3 T, B;
    tangent_basis_random(n, T, B, e2);
    const float sx = 2.0f * e0 - 1.0f;
    const float sy = 2.0f * e1 - 1.0f;
    float x = 0.0f, y = 0.0f;
    if (!(sx == 0.0f && sy == 0.0f)) {
        float r, phi;
        if (fabsf(sx) > fabsf(sy)) { r = sx; phi = (kPi / 4.0f) * (sy / fmaxf(fabsf(sx), 1e-20f)); }
        else { r = sy; phi = (kPi / 2.0f) - (kPi / 4.0f) * (sx / fmaxf(fabsf(sy), 1e-20f)); }
        float sn, cs;
        sincos_det(phi, &sn, &cs);
        x = r * cs; y = r * sn;
    }
    const float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
    const f3 dir = T * x + B * y + n * z;
    pdf = z / kPi;
    return normalize(dir);
}
__device__ __forceinline__ float fresnel_exact(float cosI, float cosT, float eta)
{
    const float invE = 1.0f / eta;
    const float rPar = (invE * cosI - cosT) / (invE * cosI + cosT);
    const float rPerp = (cosI - invE * cosT) / (cosI + invE * cosT);
    return 0.5f * (rPar * rPar + rPerp * rPerp);
}
__device__ __forceinline__ float ggx_d(float alpha, float NoH)
{
    const float a2 = alpha * alpha;
    const float d = NoH * NoH * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxf(kPi * d * d, 1e-12f);
}
__device__ __forceinline__ float ggx_g_corr(float alpha, float NoL, float NoV)
{
    const float a2 = alpha * alpha;
    const float gv = NoL * sqrtf(a2 + (1.0f - a2) * NoV * NoV);
    const float gl = NoV * sqrtf(a2 + (1.0f - a2) * NoL * NoL);
    const float den = gv + gl;
    return (den > 0.0f) ? (2.0f * NoL * NoV) / den : 0.0f;
}
__device__ __forceinline__ void ggx_params(const GB& g, float& alpha, float& kD, f3& F0)
{
    alpha = g.roughness * g.roughness;
    const float f0d = 0.08f * clampf(g.specular, 0.0f, 1.0f);
    F0 = lerp3(mk(f0d, f0d, f0d), g.albedo, g.metallic);
    kD = 1.0f - g.metallic;
}
// SampleGGXBoundedVNDF (sample.cuh:179-222)
__device__ __forceinline__ f3 sample_ggx_vndf(f3 V, f3 N, float alpha, float r0, float r1, float r2, float& pdf)
{
    f3 X, Y;
    tangent_basis_random(N, X, Y, r2);
    const float XoV = dot(X, V), YoV = dot(Y, V), NoV = dot(N, V);
    const f3 localV = mk(XoV, YoV, NoV);
    const float NoV2 = fminf(1.0f, NoV * NoV);
    const float a2 = alpha * alpha;
    const f3 lstd = mk(XoV * alpha, YoV * alpha, NoV) / sqrtf(a2 + (1.0f - a2) * NoV2);
    const float phi = 2.0f * kPi * r0;
    const float sv = 1.0f + sqrtf(1.0f - NoV2);
    const float s2 = sv * sv;
    const float k = (1.0f - a2) * s2 / (s2 + a2 * NoV2);
    const float b = NoV > 0 ? k * lstd.z : lstd.z;
    const float z = fmaf(1.0f - r1, 1.0f + b, -b);
    const float sinT = sqrtf(saturate(1.0f - z * z));
    float sp, cp;
    sincos_det(phi, &sp, &cp);
    const f3 ostd = mk(sinT * cp, sinT * sp, z);
    const f3 mstd = lstd + ostd;
    const f3 lh = normalize(mk(mstd.x * alpha, mstd.y * alpha, mstd.z));
    const f3 ll = reflect(-localV, lh);
    const f3 dir = X * ll.x + Y * ll.y + N * ll.z;
    const float ndf = ggx_d(alpha, lh.z);
    const float len2 = (1.0f - NoV2) * a2;
    const float t = sqrtf(len2 + NoV2);
    pdf = ndf / (2.0f * (k * NoV + t));
    return dir;
}
// GGXBoundedVNDF_PDF (sample.cuh:224-248)
__device__ __forceinline__ float ggx_vndf_pdf(f3 V, f3 N, f3 L, float alpha)
{
    const float NoV = dot(N, V), NoL = dot(N, L);
    if (NoV <= 0.0f || NoL <= 0.0f) return 0.0f;
    const f3 H = normalize(V + L);
    const float NoV2 = fminf(1.0f, NoV * NoV);
    const float a2 = alpha * alpha;
    const float sv = 1.0f + sqrtf(1.0f - NoV2);
    const float s2 = sv * sv;
    const float k = (1.0f - a2) * s2 / (s2 + a2 * NoV2);
    const float NoH = fmaxf(0.0f, dot(N, H));
    const float ndf = ggx_d(alpha, NoH);
    const float len2 = (1.0f - NoV2) * a2;
    const float t = sqrtf(len2 + NoV2);
    return fmaxf(ndf / (2.0f * (k * NoV + t)), 1e-12f);
}

// EvaluateBSDFWithCos, RGB (material.cuh:48-175)
__device__ __forceinline__ f3 eval_bsdf_cos(int model, f3 rayDir, f3 L, f3 N, f3 pos, const GB& g, bool inside, f3 vloc)
{
    const float NoL = fmaxf(0.0f, dot(N, L));
    if (model == AR_MAT_DIFFUSE) return g.albedo * (NoL / kPi);
    if (model == AR_MAT_GGX) {
        const f3 V = normalize(-rayDir);
        const float NoV = fmaxf(0.0f, dot(N, V));
        if (NoV <= 0.0f || NoL <= 0.0f) return mk(0.0f, 0.0f, 0.0f);
        float alpha, kD;
        f3 F0;
        ggx_params(g, alpha, kD, F0);
        // GGXLambert_BRDF (brdf.cuh:96-112)
        const f3 Hn = normalize(V + L);
        const float NoH = fmaxf(0.0f, dot(N, Hn));
        const float LoH = fmaxf(0.0f, dot(L, Hn));
        const float c = clampf(1.0f - LoH, 0.0f, 1.0f);
        const float c5 = c * c * c * c * c;
        const f3 F = mk(F0.x + (1.0f - F0.x) * c5, F0.y + (1.0f - F0.y) * c5, F0.z + (1.0f - F0.z) * c5);
        const float D = ggx_d(alpha, NoH);
        const float G = ggx_g_corr(alpha, NoL, NoV);
        f3 spec = mk(0.0f, 0.0f, 0.0f);
        if (NoL > 0.0f) spec = ((F * D) * G) / fmaxf(4.0f * NoV, 1e-7f);
        const f3 omF = mk(1.0f - F.x, 1.0f - F.y, 1.0f - F.z);
        const f3 diff = ((omF * kD) * g.albedo) * (NoL / kPi);
        return spec + diff;
    }
    if (model == AR_MAT_GLASS) {
        const float IOR = g.ior;
        f3 tr = mk(1.0f, 1.0f, 1.0f);
        if (inside) {
            // BeerLambert (brdf.cuh:15-18)
            const float dd = length(vloc - pos);
            const f3 al = vmin(vmaxs(g.albedo, 1.0e-12f), mk(1.0f, 1.0f, 1.0f));
            const float ds = dd * g.sigma_a;
            tr = mk(exp_det(ds * log_det(al.x)), exp_det(ds * log_det(al.y)), exp_det(ds * log_det(al.z)));
        }
        const f3 nIn = (dot(N, rayDir) > 0.0f) ? -N : N;
        const float eta = inside ? IOR : 1.0f / IOR;
        const float cosI = -dot(nIn, rayDir);
        const float sin2I = fmaxf(0.0f, 1.0f - cosI * cosI);
        const float k = 1.0f - sin2I * (eta * eta);
        if (k <= 0.0f) return tr * 0.99f;
        const float cosT = sqrtf(k);
        const float Fr = fresnel_exact(cosI, cosT, eta);
        const f3 R = reflect(rayDir, nIn);
        const f3 T = refract(rayDir, nIn, eta);
        const float dR = dot(L, R), dT = dot(L, T);
        if (dR >= dT) return tr * Fr;
        const float weight = (eta * eta) * (fabsf(cosT) / fmaxf(1e-6f, cosI));
        return (tr * (1.0f - Fr)) * weight;
    }
    return mk(0.0f, 0.0f, 0.0f);
}

// BSDF_PDF, RGB (material.cuh:332-387)
__device__ __forceinline__ float bsdf_pdf(int model, const GB& g, f3 N, f3 rayDir, f3 L)
{
    const f3 V = -rayDir;
    const float NoL = fmaxf(0.0f, dot(N, L));
    if (model == AR_MAT_DIFFUSE) return NoL > 0.0f ? (NoL * (1.0f / kPi)) : 0.0f;
    if (model == AR_MAT_GGX) {
        const float NoV = fmaxf(0.0f, dot(N, V));
        if (NoV <= 0.0f || NoL <= 0.0f) return 0.0f;
        float alpha, kD;
        f3 F0;
        ggx_params(g, alpha, kD, F0);
        const float pSpec = ggx_pspec(g, F0);
        const float pdfSpec = ggx_vndf_pdf(V, N, L, alpha);
        const float pdfDiff = NoL * (1.0f / kPi);
        return fmaxf(0.0f, pSpec * pdfSpec + (1.0f - pSpec) * pdfDiff);
    }
    return 0.0f;
}

__device__ __forceinline__ float power_heuristic(float pA, float pB)
{
    const float a = pA * pA, b = pB * pB;
    return a / fmaxf(1e-24f, a + b);
}

__device__ __forceinline__ float area_to_solid_angle(f3 sp, f3 lp, f3 ln, float pA)
{
    const f3 s2l = lp - sp;
    const float d2 = fmaxf(dot(s2l, s2l), 1e-20f);
    const f3 dir = s2l * rsqrt_ieee(d2);
    const float cosY = fmaxf(0.0f, dot(ln, -dir));
    if (cosY <= 0.0f) return 0.0f;
    return pA * (d2 / cosY);
}

struct Box6 {
    f3 fn[6], fc[6];
    float s1[6], s2[6], area[6];
    f3 ux, uy, uz;
};
__device__ __forceinline__ void box_facets(const Analytic& an, Box6& b)
{
    const m3 M = load_m3(an.o2w);
    b.ux = normalize(mk(M.x.x, M.y.x, M.z.x));
    b.uy = normalize(mk(M.x.y, M.y.y, M.z.y));
    b.uz = normalize(mk(M.x.z, M.y.z, M.z.z));
    const f3 c = mk(an.center[0], an.center[1], an.center[2]);
    const f3 e = mk(an.extent[0], an.extent[1], an.extent[2]);
    b.fn[0] = b.ux; b.fn[1] = -b.ux; b.fn[2] = b.uy; b.fn[3] = -b.uy; b.fn[4] = b.uz; b.fn[5] = -b.uz;
    b.fc[0] = c + b.ux * e.x; b.fc[1] = c - b.ux * e.x;
    b.fc[2] = c + b.uy * e.y; b.fc[3] = c - b.uy * e.y;
    b.fc[4] = c + b.uz * e.z; b.fc[5] = c - b.uz * e.z;
    b.s1[0] = e.y; b.s1[1] = e.y; b.s1[2] = e.x; b.s1[3] = e.x; b.s1[4] = e.x; b.s1[5] = e.x;
    b.s2[0] = e.z; b.s2[1] = e.z; b.s2[2] = e.z; b.s2[3] = e.z; b.s2[4] = e.y; b.s2[5] = e.y;
#pragma unroll
    for (int f = 0; f < 6; ++f) b.area[f] = 4.0f * b.s1[f] * b.s2[f];
}
__device__ __forceinline__ float facing_weight(f3 fn, f3 fc, f3 sp, float area)
{
    const f3 l2s = normalize(sp - fc);
    return area * fmaxf(0.0f, dot(fn, l2s));
}

// NEEPDFOmegaFromHit (nee.cuh:64-151, 254-271, 313-327)
// Face normal of light triangle l, turned towards the point p.
__device__ __forceinline__ f3 light_tri_normal(const SceneView& s, int l, f3 p, f3 lp)
{
    const float4 b = s.light_tri[3 * l + 1], c = s.light_tri[3 * l + 2];
    const f3 n = normalize(cross(mk(b.x, b.y, b.z), mk(c.x, c.y, c.z)));
    return dot(n, p - lp) < 0.0f ? -n : n;
}

__device__ float pdf_light_from_hit(const SceneView& s, int obj, f3 sp, f3 lp, f3 ln, bool tri = false)
{
    const ObjInfo oi = s.objects[obj];
    const float sel = s.light_prob[oi.light];
    if (tri && oi.type == AR_OBJ_TRIANGLE) {  // extension: triangle lights, uniform area density
        const float area = s.light_tri[3 * oi.light].w;
        if (!(area > 0.0f)) return 0.0f;
        return area_to_solid_angle(sp, lp, light_tri_normal(s, oi.light, sp, lp), sel * (1.0f / area));
    }
    if (oi.type == AR_OBJ_CUBE) {
        const Analytic& an = s.analytic[oi.aux];
        Box6 b;
        box_facets(an, b);
        int hitFacet = -1;
        for (int f = 0; f < 6; ++f) if (dot(b.fn[f], ln) > 0.999f) { hitFacet = f; break; }
        if (hitFacet < 0) {
            float best = 1e30f;
            for (int f = 0; f < 6; ++f) {
                const float dd = fabsf(dot(b.fn[f], lp - b.fc[f]));
                if (dd < best) { best = dd; hitFacet = f; }
            }
        }
        float sum = 0.0f, wHit = 0.0f, aHit = 0.0f;
        for (int f = 0; f < 6; ++f) {
            const float w = facing_weight(b.fn[f], b.fc[f], sp, b.area[f]);
            sum += w;
            if (f == hitFacet) { wHit = w; aHit = b.area[f]; }
        }
        if (sum <= 0.0f || wHit <= 0.0f) return 0.0f;
        const float pA = sel * (1.0f / aHit) * (wHit / sum);
        return area_to_solid_angle(sp, lp, ln, pA);
    }
    if (oi.type == AR_OBJ_SPHERE) {
        const Analytic& an = s.analytic[oi.aux];
        const f3 c = mk(an.center[0], an.center[1], an.center[2]);
        const float R = an.radius;
        const float dist = length(sp - c);
        if (dist <= R) return 0.0f;
        const float cosC = clampf(R / dist, 0.0f, 1.0f);
        const float areaCap = 2.0f * kPi * R * R * (1.0f - cosC);
        if (areaCap <= 1e-20f) return 0.0f;
        return area_to_solid_angle(sp, lp, ln, sel / areaCap);
    }
    return 0.0f;
}

struct LightSample {
    f3 p, n, emis;
    float pFacet, pA;
    bool valid;
};

// NEESampleLight (nee.cuh:330-377) with the box and sphere samplers
__device__ LightSample sample_light(const SceneView& s, f3 sp, Rng& g, bool tri = false)
{
    LightSample ls;
    ls.valid = false;
    if (s.num_lights <= 0) return ls;
    int pick = s.num_lights - 1;
    float pprob = 0.0f;
    {
        const float rr = g.next();
        float acc = 0.0f;
        for (int l = 0; l < s.num_lights; ++l) {
            const float p = s.light_prob[l];
            acc += p;
            if (rr < acc) { pick = l; pprob = p; break; }
        }
    }
    const int lobj = s.light_object[pick];
    const ObjInfo oi = s.objects[lobj];
    const MaterialRec& mr = s.materials[oi.material];
    if (oi.type == AR_OBJ_CUBE) {
        const Analytic& an = s.analytic[oi.aux];
        Box6 b;
        box_facets(an, b);
        int vi[6];
        float vw[6];
        int nv = 0;
        float wsum = 0.0f;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const float w = facing_weight(b.fn[f], b.fc[f], sp, b.area[f]);
            if (w > 0.0f) { vi[nv] = f; vw[nv] = w; wsum += w; ++nv; }
        }
        if (nv == 0) return ls;
        int slot = 0, fi = vi[0];
        {
            const float r = g.next() * wsum;
            float acc = 0.0f;
            for (int k = 0; k < nv; ++k) {
                acc += vw[k];
                if (r <= acc) { slot = k; fi = vi[k]; break; }
            }
        }
        const float u1 = 2.0f * g.next() - 1.0f;
        const float u2 = 2.0f * g.next() - 1.0f;
        const f3 ft = (fi < 2) ? b.uy : b.ux;
        const f3 fb = (fi < 4) ? b.uz : b.uy;
        ls.p = b.fc[fi] + ft * (u1 * b.s1[fi]) + fb * (u2 * b.s2[fi]);
        ls.n = b.fn[fi];
        ls.emis = mk(mr.emissive[0], mr.emissive[1], mr.emissive[2]);
        ls.pFacet = 1.0f * (vw[slot] / wsum);
        ls.pA = 1.0f / b.area[fi];
        ls.valid = true;
    } else if (tri && oi.type == AR_OBJ_TRIANGLE) {
        // extension: uniform point on the triangle (square-root warp of two
        // uniforms), two-sided emitter
        const float4 a = s.light_tri[3 * pick], b = s.light_tri[3 * pick + 1], c = s.light_tri[3 * pick + 2];
        if (!(a.w > 0.0f)) return ls;
        const float u1 = g.next(), u2 = g.next();
        const float su = sqrtf(u1);
        ls.p = mk(a.x, a.y, a.z) + mk(b.x, b.y, b.z) * (su * (1.0f - u2)) + mk(c.x, c.y, c.z) * (su * u2);
        ls.n = light_tri_normal(s, pick, sp, ls.p);
        ls.emis = mk(mr.emissive[0], mr.emissive[1], mr.emissive[2]);
        ls.pFacet = 1.0f;
        ls.pA = 1.0f / a.w;
        ls.valid = true;
    } else if (oi.type == AR_OBJ_SPHERE) {
        const Analytic& an = s.analytic[oi.aux];
        const f3 c = mk(an.center[0], an.center[1], an.center[2]);
        const float R = an.radius;
        const f3 p2c = sp - c;
        const float dist = length(p2c);
        if (dist <= R) return ls;
        const f3 axis = p2c / dist;
        const float cosC = clampf(R / dist, 0.0f, 1.0f);
        const float areaCap = 2.0f * kPi * R * R * (1.0f - cosC);
        const float u = g.next();
        const float vphi = g.next();
        const float cosT = lerpf(cosC, 1.0f, u);
        const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
        const float phi = 2.0f * kPi * vphi;
        f3 t, b;
        tangent_basis(axis, t, b);
        float sn, cs;
        sincos_det(phi, &sn, &cs);
        const f3 n = t * (cs * sinT) + b * (sn * sinT) + axis * cosT;
        ls.p = c + n * R;
        ls.n = n;
        ls.emis = mk(mr.emissive[0], mr.emissive[1], mr.emissive[2]);
        ls.pFacet = 1.0f;
        ls.pA = 1.0f / areaCap;
        ls.valid = true;
    } else {
        return ls;
    }
    ls.pFacet = ls.pFacet * pprob;
    return ls;
}

// SkyLighting (render.cuh:58-73)
__device__ __forceinline__ f3 sky_lighting(f3 d, int sky)
{
    if (!sky) return mk(0.0f, 0.0f, 0.0f);
    const f3 white = mk(1.0f, 1.0f, 1.0f);
    const f3 blue = mk(0.05f, 0.45f, 1.0f);
    const f3 down = mk(0.2f, 0.6f, 1.0f) * 0.125f;
    const f3 inner = lerp3(blue, white, pow_det(fmaxf(d.y, 0.0f), 0.75f));
    return lerp3(inner, down, fminf(fmaxf(-d.y * 0.5f + 0.5f, 0.0f), 1.0f)) * 0.5f;
}

}  // namespace ar
