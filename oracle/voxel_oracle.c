/*
 * CPU oracle of the triangle-surface voxelizer -- TEST INFRASTRUCTURE ONLY
 * (see lbm_oracle.h): the checker the CUDA voxelizer is compared against.
 *
 * Restates the reference's cfd::lbm::voxelize_surface and transform_surface
 * (src/lbm/voxelize.cpp:4-6): cell (i, j, k) of an nx x ny x nz grid over
 * [lo, hi] is solid when the ray from
 *     o = (lo.x + (i + 0.5) dx, lo.y + (j + 0.5) dy + 1e-10 dx, lo.z + (k + 0.5) dz + 2e-10 dx)
 * in direction +x hits an odd number of triangles, a hit being a
 * Moller-Trumbore intersection with |det| >= 1e-12, u in [0, 1], v >= 0,
 * u + v <= 1 and distance > 1e-10.  Every expression keeps the reference's
 * operand order in FP64 (built with -ffp-contract=off), so the mask equals
 * the reference's bit for bit; tests/test_voxelize_oracle.py pins it against
 * the reference compiled from its sources (oracle/_ref).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

typedef struct { double x, y, z; } vec3;

static vec3 v_sub(vec3 a, vec3 b) { vec3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static vec3 v_add(vec3 a, vec3 b) { vec3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static vec3 v_scale(vec3 a, double s) { vec3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static double v_dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static vec3 v_cross(vec3 a, vec3 b) {
    vec3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static vec3 v_load(const double* p) { vec3 r = {p[0], p[1], p[2]}; return r; }

/* Does the +x ray from o hit triangle (a, b, c)? */
static int ray_x_hits(vec3 o, vec3 a, vec3 b, vec3 c) {
    const vec3 d = {1.0, 0.0, 0.0};
    const vec3 e1 = v_sub(b, a), e2 = v_sub(c, a);
    const vec3 h = v_cross(d, e2);
    const double det = v_dot(e1, h);
    if (fabs(det) < 1e-12) return 0;
    const double inv = 1.0 / det;
    const vec3 s = v_sub(o, a);
    const double u = inv * v_dot(s, h);
    if (u < 0.0 || u > 1.0) return 0;
    const vec3 q = v_cross(s, e1);
    const double v = inv * v_dot(d, q);
    if (v < 0.0 || u + v > 1.0) return 0;
    return inv * v_dot(e2, q) > 1e-10;
}

/* mask[(k*ny + j)*nx + i] = 1 inside, 0 outside; returns 1 on invalid input
 * (no triangles, an empty grid or an empty box), as the reference throws. */
int ora_voxelize(const double* tris, size_t count, size_t nx, size_t ny, size_t nz, const double* lo,
                 const double* hi, uint8_t* mask) {
    if (count == 0 || nx == 0 || ny == 0 || nz == 0 || !(hi[0] > lo[0]) || !(hi[1] > lo[1]) || !(hi[2] > lo[2]))
        return 1;
    const double dx = (hi[0] - lo[0]) / (double)nx, dy = (hi[1] - lo[1]) / (double)ny,
                 dz = (hi[2] - lo[2]) / (double)nz;
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                const vec3 o = {lo[0] + ((double)i + 0.5) * dx, lo[1] + ((double)j + 0.5) * dy + 1e-10 * dx,
                                lo[2] + ((double)k + 0.5) * dz + 2e-10 * dx};
                size_t hits = 0;
                for (size_t t = 0; t < count; ++t) {
                    const double* p = tris + 9 * t;
                    hits += (size_t)ray_x_hits(o, v_load(p), v_load(p + 3), v_load(p + 6));
                }
                mask[(k * ny + j) * nx + i] = (uint8_t)(hits & 1U);
            }
    return 0;
}

/* Rodrigues rotation of p about `axis` (normalised here; a zero axis leaves p). */
static vec3 rotate(vec3 p, vec3 axis, double angle) {
    const double n = sqrt(v_dot(axis, axis));
    if (n < 1e-30) return p;
    axis = v_scale(axis, 1.0 / n);
    const double c = cos(angle), s = sin(angle);
    return v_add(v_add(v_scale(p, c), v_scale(v_cross(axis, p), s)), v_scale(axis, v_dot(axis, p) * (1.0 - c)));
}

/* out = every vertex rotated about `axis` by `angle`, then translated. */
int ora_transform_surface(const double* tris, size_t count, const double* translation, const double* axis,
                          double angle, double* out) {
    const vec3 tr = v_load(translation), ax = v_load(axis);
    for (size_t v = 0; v < 3 * count; ++v) {
        const vec3 r = v_add(rotate(v_load(tris + 3 * v), ax, angle), tr);
        out[3 * v] = r.x;
        out[3 * v + 1] = r.y;
        out[3 * v + 2] = r.z;
    }
    return 0;
}
