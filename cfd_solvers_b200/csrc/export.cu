// Field export: legacy-VTK structured points and the JSON live state
// (reference write_vtk_structured_3d / write_json_state_3d,
// src/lbm/visualization.cpp:39-109), and the Q-criterion of a velocity
// field (reference q_criterion_3d, :122-148) as a device kernel.
//
// ASCII files carry the same text as the reference's (17 significant digits
// for VTK, 9 for JSON: std::to_chars's general format is printf's %g, which is
// what the reference's streams print), so existing readers of its files read
// these.  Big lattices take the binary legacy format (big-endian, as the VTK
// format prescribes), which the reference does not write.
#include "export.h"

#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

namespace cfdx {
namespace {

// Buffered writer over stdio with the reference's number formatting.
class Out {
public:
    explicit Out(const std::string& path) : path_(path), f_(std::fopen(path.c_str(), "wb")) {
        if (!f_) throw std::runtime_error("cannot create " + path);
        buf_.reserve(1 << 20);
    }
    ~Out() {
        if (f_) std::fclose(f_);
    }
    Out& text(const char* s) {
        buf_.append(s);
        return spill();
    }
    Out& num(double v, int digits) {
        char tmp[64];
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, v, std::chars_format::general, digits);
        buf_.append(tmp, r.ptr);
        return spill();
    }
    Out& uint(unsigned long long v) {
        char tmp[32];
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, v);
        buf_.append(tmp, r.ptr);
        return spill();
    }
    Out& bytes(const void* p, std::size_t n) {
        buf_.append(static_cast<const char*>(p), n);
        return spill();
    }
    void close() {
        flush();
        const int rc = std::fclose(f_);
        f_ = nullptr;
        if (rc != 0) throw std::runtime_error("cannot write " + path_);
    }

private:
    Out& spill() {
        if (buf_.size() >= (1 << 20)) flush();
        return *this;
    }
    void flush() {
        if (!buf_.empty() && std::fwrite(buf_.data(), 1, buf_.size(), f_) != buf_.size())
            throw std::runtime_error("cannot write " + path_);
        buf_.clear();
    }
    std::string path_;
    std::FILE* f_;
    std::string buf_;
};

void big_endian_double(Out& o, double v) {
    std::uint64_t b;
    std::memcpy(&b, &v, 8);
    unsigned char c[8];
    for (int k = 0; k < 8; ++k) c[k] = static_cast<unsigned char>(b >> (56 - 8 * k));
    o.bytes(c, 8);
}

template <class T> __device__ __forceinline__ double load_d(const void* p, std::size_t i) {
    return double(static_cast<const T*>(p)[i]);
}

// Divisor 2 d of one axis.  When it is a power of two, x / (2 d) and
// x * (1 / (2 d)) are correctly rounded values of the same real number, so the
// kernel multiplies (one instruction instead of a division sequence).
struct Spacing {
    double d2, inv;
    int pow2;
};

__device__ __forceinline__ double by_spacing(double x, const Spacing& s) {
    return s.pow2 ? __dmul_rn(x, s.inv) : __ddiv_rn(x, s.d2);
}

// The reference's central-difference gradient and Q = (|Omega|^2 - |S|^2)/2,
// operand for operand in FP64 without contraction; the outer layer of the grid is 0.
// Terms that are equal in IEEE arithmetic are computed once (s_ji = s_ij,
// o_ji^2 = o_ij^2, s_ii = g_ii, o_ii = +0 adds nothing), with the reference's
// order of additions kept, so the result is the nine-term loop's bit for bit.
template <class T>
__global__ void __launch_bounds__(128) k_q_criterion(const void* ux, const void* uy, const void* uz,
                                                     std::size_t stride, std::uint32_t nx, std::uint32_t ny,
                                                     std::uint32_t nz, Spacing hx, Spacing hy, Spacing hz, double* q) {
    const std::uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    const std::size_t n = (std::size_t(z) * ny + y) * nx + x;
    if (x == 0 || y == 0 || z == 0 || x + 1 >= nx || y + 1 >= ny || z + 1 >= nz) {
        q[n] = 0.0;
        return;
    }
    const std::size_t sx = 1, sy = nx, sz = std::size_t(nx) * ny;
    const void* u[3] = {ux, uy, uz};
    double g[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        g[c][0] = by_spacing(__dsub_rn(load_d<T>(u[c], (n + sx) * stride), load_d<T>(u[c], (n - sx) * stride)), hx);
        g[c][1] = by_spacing(__dsub_rn(load_d<T>(u[c], (n + sy) * stride), load_d<T>(u[c], (n - sy) * stride)), hy);
        g[c][2] = by_spacing(__dsub_rn(load_d<T>(u[c], (n + sz) * stride), load_d<T>(u[c], (n - sz) * stride)), hz);
    }
    double ss[3][3], oo[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        ss[i][i] = __dmul_rn(g[i][i], g[i][i]);
#pragma unroll
        for (int j = i + 1; j < 3; ++j) {
            const double sij = __dmul_rn(0.5, __dadd_rn(g[i][j], g[j][i]));
            const double oij = __dmul_rn(0.5, __dsub_rn(g[i][j], g[j][i]));
            ss[i][j] = ss[j][i] = __dmul_rn(sij, sij);
            oo[i][j] = oo[j][i] = __dmul_rn(oij, oij);
        }
    }
    double s2 = 0.0, o2 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            s2 = __dadd_rn(s2, ss[i][j]);
            if (i != j) o2 = __dadd_rn(o2, oo[i][j]);
        }
    q[n] = __dmul_rn(0.5, __dsub_rn(o2, s2));
}

Spacing spacing(double d) {
    Spacing s{2 * d, 0.0, 0}; // 2 * d as the reference writes it: exact for every finite d
    int e = 0;
    if (std::isfinite(s.d2) && s.d2 > 0.0 && std::frexp(s.d2, &e) == 0.5) {
        s.inv = std::ldexp(1.0, 1 - e); // 2 d = 2^(e-1)
        s.pow2 = std::isnormal(s.inv) ? 1 : 0;
    }
    return s;
}

} // namespace

void write_vtk_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz, const double* scalar,
                  const double* velocity, const std::uint8_t* solid, const char* name, bool binary) {
    const std::size_t cells = nx * ny * nz;
    if (nx == 0 || ny == 0 || nz == 0 || !scalar || !path || !name)
        throw std::invalid_argument("LBM 3-D VTK field size mismatch");
    Out o(path);
    o.text("# vtk DataFile Version 3.0\ncfd_solvers LBM 3-D\n").text(binary ? "BINARY" : "ASCII");
    o.text("\nDATASET STRUCTURED_POINTS\nDIMENSIONS ").uint(nx).text(" ").uint(ny).text(" ").uint(nz);
    o.text("\nORIGIN 0 0 0\nSPACING 1 1 1\nPOINT_DATA ").uint(cells).text("\nSCALARS ").text(name);
    o.text(" double 1\nLOOKUP_TABLE default\n");
    if (binary) {
        for (std::size_t i = 0; i < cells; ++i) big_endian_double(o, scalar[i]);
        o.text("\n");
    } else {
        for (std::size_t i = 0; i < cells; ++i) o.num(scalar[i], 17).text("\n");
    }
    if (velocity) {
        o.text("VECTORS velocity double\n");
        if (binary) {
            for (std::size_t i = 0; i < 3 * cells; ++i) big_endian_double(o, velocity[i]);
            o.text("\n");
        } else {
            for (std::size_t i = 0; i < cells; ++i)
                o.num(velocity[3 * i], 17).text(" ").num(velocity[3 * i + 1], 17).text(" ").num(velocity[3 * i + 2], 17)
                    .text("\n");
        }
    }
    if (solid) {
        o.text("SCALARS solid unsigned_char 1\nLOOKUP_TABLE default\n");
        if (binary) {
            o.bytes(solid, cells);
            o.text("\n");
        } else {
            for (std::size_t i = 0; i < cells; ++i) o.uint(solid[i]).text("\n");
        }
    }
    o.close();
}

void write_json_state_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz, std::uint64_t step,
                         const double* scalar, const std::uint8_t* solid, const char* name) {
    const std::size_t cells = nx * ny * nz;
    if (nx == 0 || ny == 0 || nz == 0 || !scalar || !path || !name)
        throw std::invalid_argument("LBM 3-D live state size mismatch");
    const std::string tmp = std::string(path) + ".tmp";
    {
        Out o(tmp);
        o.text("{\n  \"dimensions\": [").uint(nx).text(", ").uint(ny).text(", ").uint(nz).text("],\n  \"step\": ");
        o.uint(step).text(",\n  \"field\": \"").text(name).text("\",\n  \"values\": [");
        for (std::size_t i = 0; i < cells; ++i) {
            if (i) o.text(", ");
            o.num(scalar[i], 9);
        }
        o.text("]");
        if (solid) {
            o.text(",\n  \"solid\": [");
            for (std::size_t i = 0; i < cells; ++i) {
                if (i) o.text(", ");
                o.uint(solid[i]);
            }
            o.text("]");
        }
        o.text("\n}\n");
        o.close();
    }
    // publish atomically where the file system allows (readers poll this file)
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(path);
        if (std::rename(tmp.c_str(), path) != 0)
            throw std::runtime_error(std::string("cannot publish 3-D LBM live state: ") + path);
    }
}

cudaError_t launch_q_criterion(const void* ux, const void* uy, const void* uz, bool f64, std::size_t stride,
                               std::size_t nx, std::size_t ny, std::size_t nz, double dx, double dy, double dz,
                               double* q, cudaStream_t s) {
    const dim3 grid(static_cast<unsigned>((nx + 127) / 128), static_cast<unsigned>(ny), static_cast<unsigned>(nz));
    const Spacing hx = spacing(dx), hy = spacing(dy), hz = spacing(dz);
    if (f64)
        k_q_criterion<double><<<grid, 128, 0, s>>>(ux, uy, uz, stride, std::uint32_t(nx), std::uint32_t(ny),
                                                   std::uint32_t(nz), hx, hy, hz, q);
    else
        k_q_criterion<float><<<grid, 128, 0, s>>>(ux, uy, uz, stride, std::uint32_t(nx), std::uint32_t(ny),
                                                  std::uint32_t(nz), hx, hy, hz, q);
    return cudaGetLastError();
}

} // namespace cfdx
