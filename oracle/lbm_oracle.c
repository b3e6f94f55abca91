/*
 * CPU oracle for the in-place Esoteric-Pull step -- TEST INFRASTRUCTURE ONLY.
 * See lbm_oracle.h for scope and the reference files it restates.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).  Contraction
 * must stay off: the FP32 variant is pinned bit for bit against the reference
 * compiled with the same flag.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Velocity sets in the reference's order: pairs (2p+1, 2p+2) are opposite
 * (include/cfd/solvers/lbm/descriptors.hpp:59-146).  The order has to match
 * the reference so that logical populations compare index for index. */
typedef struct {
    int q;
    int cx[27], cy[27], cz[27];
    int opp[27];
    float wf[27];
    double wd[27];
} ora_lattice;

static const int k_cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
static const int k_cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
static const int k_cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};

static void ora_make_lattice(int q, ora_lattice* L) {
    L->q = q;
    for (int d = 0; d < 27; ++d) {
        L->cx[d] = k_cx[d];
        L->cy[d] = k_cy[d];
        L->cz[d] = k_cz[d];
        L->opp[d] = d == 0 ? 0 : ((d & 1) ? d + 1 : d - 1);
    }
    for (int d = 0; d < q; ++d) {
        const int len2 = k_cx[d] * k_cx[d] + k_cy[d] * k_cy[d] + k_cz[d] * k_cz[d];
        if (q == 19) {
            L->wf[d] = len2 == 0 ? 1.0F / 3.0F : (len2 == 1 ? 1.0F / 18.0F : 1.0F / 36.0F);
            L->wd[d] = len2 == 0 ? 1.0 / 3.0 : (len2 == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
        } else {
            L->wf[d] = len2 == 0 ? 8.0F / 27.0F
                                 : (len2 == 1 ? 2.0F / 27.0F : (len2 == 2 ? 1.0F / 54.0F : 1.0F / 216.0F));
            L->wd[d] = len2 == 0 ? 8.0 / 27.0 : (len2 == 1 ? 2.0 / 27.0 : (len2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
        }
    }
}

/* esoteric_pull.hpp:40-46,304-310 */
static size_t ora_shift(size_t c, int delta, size_t extent) {
    if (delta > 0) return c + 1U == extent ? 0U : c + 1U;
    if (delta < 0) return c == 0U ? extent - 1U : c - 1U;
    return c;
}

static size_t ora_neighbor(const ora_cfg* c, size_t x, size_t y, size_t z, int dx, int dy, int dz) {
    const size_t xn = ora_shift(x, dx, c->nx);
    const size_t yn = ora_shift(y, dy, c->ny);
    const size_t zn = ora_shift(z, dz, c->nz);
    return (zn * c->ny + yn) * c->nx + xn;
}

/* IEEE 754 binary32 -> binary16, round to nearest, ties to even. */
uint16_t ora_f32_to_f16(float v) {
    uint32_t b;
    memcpy(&b, &v, sizeof b);
    const uint32_t sign = (b >> 16) & 0x8000U;
    const uint32_t exp = (b >> 23) & 0xffU;
    uint32_t man = b & 0x7fffffU;
    if (exp == 0xffU) return (uint16_t)(sign | 0x7c00U | (man ? 0x200U : 0U));
    const int e = (int)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00U);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        man |= 0x800000U;
        const int shift = 14 - e;
        uint32_t h = man >> shift;
        const uint32_t rem = man & ((1U << shift) - 1U);
        const uint32_t half = 1U << (shift - 1);
        if (rem > half || (rem == half && (h & 1U))) ++h;
        return (uint16_t)(sign | h);
    }
    uint32_t h = sign | ((uint32_t)e << 10) | (man >> 13);
    const uint32_t rem = man & 0x1fffU;
    if (rem > 0x1000U || (rem == 0x1000U && (h & 1U))) ++h;
    return (uint16_t)h;
}

float ora_f16_to_f32(uint16_t h) {
    const uint32_t sign = ((uint32_t)h & 0x8000U) << 16;
    const uint32_t exp = ((uint32_t)h >> 10) & 0x1fU;
    const uint32_t man = (uint32_t)h & 0x3ffU;
    uint32_t b;
    if (exp == 0U) {
        const float v = ldexpf((float)man, -24);
        return sign ? -v : v;
    }
    if (exp == 31U)
        b = sign | 0x7f800000U | (man << 13);
    else
        b = sign | ((exp - 15U + 127U) << 23) | (man << 13);
    float v;
    memcpy(&v, &b, sizeof v);
    return v;
}

float ora_reference_les_k(void) {
    const float pi = 3.14159265358979323846F;
    return 16.0F * 1.4142135623730950488F / (3.0F * pi * pi);
}

/* ---- FP32 storage, FP32 arithmetic ---- */
#define REAL float
#define STORE float
#define MACRO_T float
#define SFX(name) name##_f32
#define R(x) x##F
#define W(d) (L->wf[d])
#define SQRT sqrtf
#define SIN sinf
#define COS cosf
#define ORA_PI(T) 3.14159265358979323846F
#define LOADP(d, m) (f[(size_t)(d) * N + (m)])
#define STOREP(d, m, v) (f[(size_t)(d) * N + (m)] = (v))
#include "lbm_oracle_body.inc"
#undef REAL
#undef STORE
#undef MACRO_T
#undef SFX
#undef R
#undef W
#undef SQRT
#undef SIN
#undef COS
#undef ORA_PI
#undef LOADP
#undef STOREP

/* ---- FP64 storage, FP64 arithmetic ---- */
#define REAL double
#define STORE double
#define MACRO_T double
#define SFX(name) name##_f64
#define R(x) x
#define W(d) (L->wd[d])
#define SQRT sqrt
#define SIN sin
#define COS cos
#define ORA_PI(T) 3.14159265358979323846
#define LOADP(d, m) (f[(size_t)(d) * N + (m)])
#define STOREP(d, m, v) (f[(size_t)(d) * N + (m)] = (v))
#include "lbm_oracle_body.inc"
#undef REAL
#undef STORE
#undef MACRO_T
#undef SFX
#undef R
#undef W
#undef SQRT
#undef SIN
#undef COS
#undef ORA_PI
#undef LOADP
#undef STOREP

/* ---- FP16 shifted storage (h = half((f - w_d) * s_d)), FP32 arithmetic ----
 * Reference codec: compressed_pull.hpp:72-79 (s_d = 1). */
static float g_scale[27], g_inv_scale[27];
#define REAL float
#define STORE uint16_t
#define MACRO_T float
#define SFX(name) name##_h16
#define R(x) x##F
#define W(d) (L->wf[d])
#define SQRT sqrtf
#define SIN sinf
#define COS cosf
#define ORA_PI(T) 3.14159265358979323846F
#define LOADP(d, m) (W(d) + ora_f16_to_f32(f[(size_t)(d) * N + (m)]) * g_inv_scale[d])
#define STOREP(d, m, v) (f[(size_t)(d) * N + (m)] = ora_f32_to_f16(((v) - W(d)) * g_scale[d]))
#include "lbm_oracle_body.inc"
#undef REAL
#undef STORE
#undef MACRO_T
#undef SFX
#undef R
#undef W
#undef SQRT
#undef SIN
#undef COS
#undef ORA_PI
#undef LOADP
#undef STOREP

static int ora_setup(const ora_cfg* c, ora_lattice* L) {
    if (!c || (c->q != 19 && c->q != 27)) return 1;
    if (c->nx < 2 || c->ny < 2 || c->nz < 2) return 1;
    if (!(c->tau > 0.5)) return 1;
    ora_make_lattice(c->q, L);
    if (c->storage == ORA_STORE_F16S) {
        for (int d = 0; d < c->q; ++d) {
            g_scale[d] = c->scale ? c->scale[d] : 1.0F;
            g_inv_scale[d] = 1.0F / g_scale[d];
        }
    }
    return 0;
}

size_t ora_population_bytes(const ora_cfg* c) {
    const size_t N = c->nx * c->ny * c->nz;
    const size_t s = c->storage == ORA_STORE_F64 ? 8U : (c->storage == ORA_STORE_F16S ? 2U : 4U);
    return (size_t)c->q * N * s;
}

int ora_init(const ora_cfg* c, void* f, int kind, const float* p, const float* fields) {
    ora_lattice L;
    if (ora_setup(c, &L)) return 1;
    if (c->storage == ORA_STORE_F32)
        init_f32(&L, c, (float*)f, kind, p, fields);
    else if (c->storage == ORA_STORE_F64)
        init_f64(&L, c, (double*)f, kind, p, fields);
    else
        init_h16(&L, c, (uint16_t*)f, kind, p, fields);
    return 0;
}

int ora_step(const ora_cfg* c, void* f, uint64_t t) { return ora_step_planes(c, f, t, 0, c ? c->nz : 0); }

int ora_step_planes(const ora_cfg* c, void* f, uint64_t t, size_t z_begin, size_t z_end) {
    ora_lattice L;
    if (ora_setup(c, &L)) return 1;
    if (z_begin > z_end || z_end > c->nz) return 1;
    if (c->storage == ORA_STORE_F32)
        step_f32(&L, c, (float*)f, t, z_begin, z_end);
    else if (c->storage == ORA_STORE_F64)
        step_f64(&L, c, (double*)f, t, z_begin, z_end);
    else
        step_h16(&L, c, (uint16_t*)f, t, z_begin, z_end);
    return 0;
}

int ora_macroscopic(const ora_cfg* c, const void* f, uint64_t t, void* rho, void* ux, void* uy, void* uz) {
    ora_lattice L;
    if (ora_setup(c, &L)) return 1;
    if (c->storage == ORA_STORE_F32)
        macroscopic_f32(&L, c, (const float*)f, t, (float*)rho, (float*)ux, (float*)uy, (float*)uz);
    else if (c->storage == ORA_STORE_F64)
        macroscopic_f64(&L, c, (const double*)f, t, (double*)rho, (double*)ux, (double*)uy, (double*)uz);
    else
        macroscopic_h16(&L, c, (const uint16_t*)f, t, (float*)rho, (float*)ux, (float*)uy, (float*)uz);
    return 0;
}

int ora_reduce(const ora_cfg* c, const void* f, uint64_t t, double out[7]) {
    ora_lattice L;
    if (ora_setup(c, &L)) return 1;
    if (c->storage == ORA_STORE_F32)
        reduce_f32(&L, c, (const float*)f, t, out);
    else if (c->storage == ORA_STORE_F64)
        reduce_f64(&L, c, (const double*)f, t, out);
    else
        reduce_h16(&L, c, (const uint16_t*)f, t, out);
    return 0;
}

int ora_logical(const ora_cfg* c, const void* f, uint64_t t, void* out) {
    ora_lattice L;
    if (ora_setup(c, &L)) return 1;
    if (c->storage == ORA_STORE_F32)
        logical_f32(&L, c, (const float*)f, t, (float*)out);
    else if (c->storage == ORA_STORE_F64)
        logical_f64(&L, c, (const double*)f, t, (double*)out);
    else
        logical_h16(&L, c, (const uint16_t*)f, t, (float*)out);
    return 0;
}
