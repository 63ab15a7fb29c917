// Output kernels: vorticity slices and the XZ plane dump, with the
// reference's excluded output points.
//
//   vorticity  calcVorticityXZ / calcVorticityXY (ComputeUnitOutput.hpp:113-285,
//              GPU ComputeUnitOutput.cuh:10-64): log |curl u|^2 from central
//              differences of u = j / rho (QVec::velocity(), QVec.hpp:136-144)
//              of the moments the reference's Q holds between steps;
//              excluded cells give -1 (the GPU kernel's value).
//   plane      savePlaneXZ<float, 4> (ComputeUnitOutput.hpp:354-447): for
//              every non-excluded cell of the plane, in (i, k) order, a
//              tDiskGrid<float, 4> record (Output.hpp:22-26) of Q slots 0..3
//              (Simple: the first four moments; Esotwist: the raw slots,
//              see k_plane_xz), and a tDiskGrid<float, 3> record of F where
//              F is non-zero.
//   exclude    setOutputExcludePoints / unsetOutputExcludePoints
//              (ComputeUnitOutput.hpp:20-53): one bit per cell.
//
// Neighbours beyond the lattice faces: the reference reads its ghost layer
// there, which its step never fills with moments (Simple: the streamed-out
// populations of the bounce-back; Esotwist: the initial values), so those
// cells' vorticity is not meaningful in the reference. Here the cell itself
// stands in for the missing neighbour.
#include "tdlb_handle.hpp"
#include "step_kernels.cuh"

#include <cstring>
#include <string>
#include <vector>

namespace tdlb {

// u = j / rho of cell (i, j, k), clamped into the lattice.
template <typename S>
__device__ __forceinline__ void cell_velocity(const Planes& A, const Dims& g, int mode, int even, const CollideParams& p,
                                              int i, int j, int k, float (&u)[3]) {
    i = min(max(i, 0), g.nx - 1);
    j = min(max(j, 0), g.ny - 1);
    k = min(max(k, 0), g.nz - 1);
    float m[NQ];
    state_moments18<S>(A, g, mode, even, p, i, j, k, m);
    u[0] = m[1] / m[0];
    u[1] = m[2] / m[0];
    u[2] = m[3] / m[0];
}

// axis 1: XZ slice at j = cut, out[i * z + k]; axis 2: XY slice at k = cut,
// out[j * x + i] (the reference's picture layouts).
template <typename S>
__global__ void __launch_bounds__(256) k_vorticity(Planes A, Dims g, int mode, int even, CollideParams p, int axis,
                                                   int cut, const uint32_t* __restrict__ excl, float* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    long long o;
    if (axis == 1) {
        if (t >= (long long)g.nx * g.nz) return;
        i = (int)(t / g.nz);
        k = (int)(t - (long long)i * g.nz);
        j = cut;
        o = (long long)i * g.nz + k;
    } else {
        if (t >= (long long)g.nx * g.ny) return;
        j = (int)(t / g.nx);
        i = (int)(t - (long long)j * g.nx);
        k = cut;
        o = (long long)j * g.nx + i;
    }
    const long long row = (long long)i * g.ny + j;
    if (excl && ((excl[row * g.kw + (k >> 5)] >> (k & 31)) & 1u)) {
        out[o] = -1.f;
        return;
    }
    float q05[3], q06[3], q03[3], q04[3], q01[3], q02[3];
    cell_velocity<S>(A, g, mode, even, p, i, j, k + 1, q05);
    cell_velocity<S>(A, g, mode, even, p, i, j, k - 1, q06);
    cell_velocity<S>(A, g, mode, even, p, i, j + 1, k, q03);
    cell_velocity<S>(A, g, mode, even, p, i, j - 1, k, q04);
    cell_velocity<S>(A, g, mode, even, p, i + 1, j, k, q01);
    cell_velocity<S>(A, g, mode, even, p, i - 1, j, k, q02);
    const float uxy = 0.5f * (q05[0] - q06[0]);
    const float uxz = 0.5f * (q03[0] - q04[0]);
    const float uyx = 0.5f * (q01[1] - q02[1]);
    const float uyz = 0.5f * (q03[1] - q04[1]);
    const float uzx = 0.5f * (q01[2] - q02[2]);
    const float uzy = 0.5f * (q05[2] - q06[2]);
    const float a = uxy - uyx, b = uyz - uzy, c = uzx - uxz;
    out[o] = logf(b * b + c * c + a * a);
}

// The XZ plane at j: Q slots 0..3 as the reference holds them, F (zero where
// the last pass did not touch the cell) and the excluded bit of every cell,
// out[(i * z + k) * 8 + l]. Simple: the cell's own first four moments.
// Esotwist: the reference's savePlaneXZ copies the raw slots of its Q, which
// after moments() hold the writeMoments placement -- slot s at location x is
// moment d = (even ? s : s^1) of cell x - max(-c_d, 0) (wrapping) -- so each
// slot is that moment of that cell.
template <typename S>
__global__ void __launch_bounds__(256) k_plane_xz(Planes A, Dims g, int mode, int even, CollideParams p, int j,
                                                  int esotwist, const float4* __restrict__ F,
                                                  const uint32_t* __restrict__ mask, const uint32_t* __restrict__ excl,
                                                  float* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.nz) return;
    const int i = (int)(t / g.nz), k = (int)(t - (long long)(t / g.nz) * g.nz);
    const long long row = (long long)i * g.ny + j;
    const long long e = row * g.kp + k;
    float* o = out + t * 8;
    float m[NQ];
    if (!esotwist) {
        state_moments18<S>(A, g, mode, even, p, i, j, k, m);
        o[0] = m[0];
        o[1] = m[1];
        o[2] = m[2];
        o[3] = m[3];
    } else {
        for (int s = 0; s < 4; s++) {
            const int d = even ? s : (s ^ 1);
            const int si = cx_of(d) < 0 ? (i == 0 ? g.nx - 1 : i - 1) : i;
            const int sj = cy_of(d) < 0 ? (j == 0 ? g.ny - 1 : j - 1) : j;
            const int sk = cz_of(d) < 0 ? (k == 0 ? g.nz - 1 : k - 1) : k;
            state_moments18<S>(A, g, mode, even, p, si, sj, sk, m);
            o[s] = m[d];
        }
    }
    const bool on = (mask[row * g.kw + (k >> 5)] >> (k & 31)) & 1u;
    const float4 v = F[e];
    o[4] = on ? v.x : 0.f;
    o[5] = on ? v.y : 0.f;
    o[6] = on ? v.z : 0.f;
    o[7] = excl && ((excl[row * g.kw + (k >> 5)] >> (k & 31)) & 1u) ? 1.f : 0.f;
}

}  // namespace tdlb

namespace {

struct OFail {
    int code;
    std::string msg;
};

#define TDLB_OCK(call)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) throw OFail{TDLB_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

template <typename F>
int oguard(tdlb_lattice* h, F&& fn) {
    if (!h) return TDLB_EINVAL;
    try {
        cudaSetDevice(h->device);
        const cudaError_t je = tdlb_rt::join_side(h);   // after every queued step and forcing pass
        if (je != cudaSuccess) throw OFail{TDLB_ECUDA, std::string("join: ") + cudaGetErrorString(je)};
        fn();
        return TDLB_OK;
    } catch (const OFail& f) {
        h->err = f.msg;
        return f.code;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return TDLB_ENOMEM;
    } catch (const std::exception& e) {
        h->err = e.what();
        return TDLB_EINVAL;
    }
}

void require(tdlb_lattice* h) {
    if (!h->initialised) throw OFail{TDLB_ESTATE, "not initialised (tdlb_initialise)"};
}

// Device scratch freed on every exit path.
struct DevBuf {
    float* p = nullptr;
    ~DevBuf() { cudaFree(p); }
};

unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

extern "C" {

int tdlb_set_output_exclude(tdlb_handle h, const tdlb_marker* markers, size_t n, int exclude) {
    return oguard(h, [&] {
        if (n && !markers) throw OFail{TDLB_EINVAL, "markers is NULL"};
        const Dims& g = h->g;
        for (size_t q = 0; q < n; q++)
            if (markers[q].i < 0 || markers[q].i >= g.nx || markers[q].j < 0 || markers[q].j >= g.ny ||
                markers[q].k < 0 || markers[q].k >= g.nz)
                throw OFail{TDLB_EINVAL, "marker " + std::to_string(q) + " outside the interior"};
        if (h->h_exclude.empty()) h->h_exclude.assign((size_t)h->mask_words, 0u);
        for (size_t q = 0; q < n; q++) {
            const long long row = markers[q].i * g.ny + markers[q].j;
            const int k = (int)markers[q].k;
            uint32_t& w = h->h_exclude[(size_t)(row * g.kw + (k >> 5))];
            if (exclude) w |= 1u << (k & 31);
            else w &= ~(1u << (k & 31));
        }
        if (!h->d_exclude) TDLB_OCK(cudaMalloc(&h->d_exclude, (size_t)h->mask_words * sizeof(uint32_t)));
        TDLB_OCK(cudaMemcpyAsync(h->d_exclude, h->h_exclude.data(), h->h_exclude.size() * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, h->stream));
        TDLB_OCK(cudaStreamSynchronize(h->stream));
    });
}

static int vorticity(tdlb_handle h, int axis, int64_t cut, float* out) {
    return oguard(h, [&] {
        require(h);
        const Dims& g = h->g;
        const long long lim = axis == 1 ? g.ny : g.nz;
        if (!out || cut < 0 || cut >= lim) throw OFail{TDLB_EINVAL, "cut outside the lattice or out is NULL"};
        const long long n = axis == 1 ? (long long)g.nx * g.nz : (long long)g.nx * g.ny;
        DevBuf d;
        TDLB_OCK(cudaMalloc(&d.p, (size_t)n * sizeof(float)));
        const Planes A = h->planes(h->state_buf());
        const int mode = h->state_mode(), even = h->even ? 1 : 0;
        tdlb::with_storage(h->cfg.storage, [&](auto s) {
            tdlb::k_vorticity<decltype(s)><<<blocks(n), 256, 0, h->stream>>>(A, g, mode, even, h->cp, axis, (int)cut,
                                                                            h->d_exclude, d.p);
        });
        TDLB_OCK(cudaGetLastError());
        TDLB_OCK(cudaMemcpyAsync(out, d.p, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        TDLB_OCK(cudaStreamSynchronize(h->stream));
    });
}

int tdlb_vorticity_xz(tdlb_handle h, int64_t j, float* out) { return vorticity(h, 1, j, out); }
int tdlb_vorticity_xy(tdlb_handle h, int64_t k, float* out) { return vorticity(h, 2, k, out); }

int tdlb_plane_xz(tdlb_handle h, int64_t j, tdlb_disk_grid4* q_out, size_t q_cap, size_t* q_n, tdlb_disk_grid3* f_out,
                  size_t f_cap, size_t* f_n) {
    return oguard(h, [&] {
        require(h);
        const Dims& g = h->g;
        if (j < 0 || j >= g.ny) throw OFail{TDLB_EINVAL, "j outside the lattice"};
        if (!q_n || !f_n) throw OFail{TDLB_EINVAL, "q_n and f_n are required"};
        const long long n = (long long)g.nx * g.nz;
        DevBuf d;
        TDLB_OCK(cudaMalloc(&d.p, (size_t)n * 8 * sizeof(float)));
        const Planes A = h->planes(h->state_buf());
        const int mode = h->state_mode(), even = h->even ? 1 : 0;
        tdlb::with_storage(h->cfg.storage, [&](auto s) {
            tdlb::k_plane_xz<decltype(s)><<<blocks(n), 256, 0, h->stream>>>(A, g, mode, even, h->cp, (int)j,
                                                                           h->cfg.streaming == TDLB_STREAMING_ESOTWIST,
                                                                           reinterpret_cast<const float4*>(h->F),
                                                                           h->mask_cur(), h->d_exclude, d.p);
        });
        TDLB_OCK(cudaGetLastError());
        std::vector<float> host((size_t)n * 8);
        TDLB_OCK(cudaMemcpyAsync(host.data(), d.p, host.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        TDLB_OCK(cudaStreamSynchronize(h->stream));
        size_t nq = 0, nf = 0;
        for (long long c = 0; c < n; c++) {
            const float* v = host.data() + c * 8;
            if (v[7] != 0.f) continue;
            const int i = (int)(c / g.nz), k = (int)(c % g.nz);
            if (q_out && nq < q_cap) {
                tdlb_disk_grid4& r = q_out[nq];
                r.iGrid = (uint16_t)i;
                r.jGrid = (uint16_t)j;        // savePlaneXZ: j - 1 in ghosted cells
                r.kGrid = (uint16_t)k;
                r.pad = 0;
                std::memcpy(r.q, v, 4 * sizeof(float));
            }
            nq++;
            if (v[4] != 0.f || v[5] != 0.f || v[6] != 0.f) {   // Force::isNotZero
                if (f_out && nf < f_cap) {
                    tdlb_disk_grid3& r = f_out[nf];
                    r.iGrid = (uint16_t)i;
                    r.jGrid = (uint16_t)(j + 1);  // savePlaneXZ writes the ghosted j for F
                    r.kGrid = (uint16_t)k;
                    r.pad = 0;
                    std::memcpy(r.q, v + 4, 3 * sizeof(float));
                }
                nf++;
            }
        }
        *q_n = nq;
        *f_n = nf;
        if ((q_out && nq > q_cap) || (f_out && nf > f_cap)) throw OFail{TDLB_EINVAL, "output capacity too small"};
    });
}

}  // extern "C"
