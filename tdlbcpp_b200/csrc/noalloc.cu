// tdlb_impeller_load_noalloc: the FP64 impeller load without any allocation.
//
// Who needs it: callers that cannot allocate device memory once their
// simulation is running -- a host application that hands all GPU memory to
// its own pool up front (a cudaMalloc from the library would fail or escape
// the pool's accounting), or a real-time loop with a no-allocation rule after
// start-up (cudaMalloc can synchronise the device and has no time bound).
// The allocating entry point, tdlb_impeller_load, creates its reduction
// buffer with cudaMalloc on its first call; this variant keeps that buffer
// in a fixed-size array compiled into the library instead.
//
// The scratch: g_load_partials below, a file-scope __device__ array of
// kNoAllocMaxBlocks * 5 doubles (40 KiB). Every GPU that loads the library
// holds it until the process exits. It bounds the number of markers this
// entry point accepts to kNoAllocMaxBlocks * kNoAllocChunk (1,048,576);
// larger lists are rejected with TDLB_EINVAL.
//
// Sharing: every call on a device uses the same array, and the array keeps
// what the last call left in it. Each call overwrites every partial it
// later reads, so nothing needs clearing, but two calls whose work overlaps
// on the GPU (different streams, or different handles on one device without
// ordering between them) race on the array.
//
// Set-up: the host cannot use the array's name as a device address. The
// first call on each device looks the address up with cudaGetSymbolAddress
// (with that device current) and keeps it; make that first call before any
// stream capture starts. A device reset (cudaDeviceReset) in the same
// process invalidates the kept address, and a later call would write through
// it: do not call this entry point after a reset.
#include "tdlb_handle.hpp"

#include <mutex>

namespace {

constexpr int kNoAllocChunk = 1024;        // markers summed by one block
constexpr int kNoAllocMaxBlocks = 1024;    // blocks the array has room for
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_load_partials[kNoAllocMaxBlocks * 5];

std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {};

// Block b sums slots [b*1024, b*1024 + 1024) in a fixed order (4 per thread,
// then a shared-memory tree), so the result does not depend on timing.
__global__ void __launch_bounds__(256) k_marker_load_chunks(const float* __restrict__ sums,
                                                            const int* __restrict__ sched,
                                                            const tdlb::Marker* __restrict__ markers, int n,
                                                            int begin, float beta, double ci, double ck,
                                                            double* __restrict__ partial) {
    __shared__ double red[5][256];
    double acc[5] = {0, 0, 0, 0, 0};
    const int base = blockIdx.x * kNoAllocChunk;
    for (int t = 0; t < kNoAllocChunk / 256; t++) {
        const int p = base + t * 256 + threadIdx.x;
        if (p >= n) break;
        const int q = sched[p];
        if (q < begin) continue;
        const tdlb::Marker mk = markers[q];
        const double fx = -(double)beta * (double)sums[p];
        const double fy = -(double)beta * (double)sums[n + p];
        const double fz = -(double)beta * (double)sums[2 * n + p];
        const double di = (double)mk.i + (double)mk.iCartFraction - ci;
        const double dk = (double)mk.k + (double)mk.kCartFraction - ck;
        acc[0] += fx;
        acc[1] += fy;
        acc[2] += fz;
        acc[3] += dk * fx - di * fz;
        acc[4] += 1.0;
    }
    for (int c = 0; c < 5; c++) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 5; c++) red[c][threadIdx.x] += red[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 5; c++) partial[blockIdx.x * 5 + c] = red[c][0];
}

__global__ void k_marker_load_chunks_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < nblocks; b++)
        for (int c = 0; c < 5; c++) acc[c] += partial[b * 5 + c];
    for (int c = 0; c < 5; c++) out[c] = acc[c];
}

// Device address of g_load_partials on the current device (looked up once).
cudaError_t partials_address(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_load_partials);
        if (e != cudaSuccess) return e;
        g_addr[device] = static_cast<double*>(p);
    }
    *out = g_addr[device];
    return cudaSuccess;
}

// Error text without allocating (the handle reserves room for messages).
int fail(tdlb_lattice* h, int code, const char* msg) {
    h->err.assign(msg);
    return code;
}

}  // namespace

extern "C" int tdlb_impeller_load_noalloc(tdlb_handle h, double* d_out5) {
    if (!h) return TDLB_EINVAL;
    if (!d_out5) return fail(h, TDLB_EINVAL, "d_out5 is NULL");
    if (h->impeller_begin < 0) return fail(h, TDLB_ESTATE, "no impeller attached (tdlb_attach_rushton)");
    if (h->pass == 0) return fail(h, TDLB_ESTATE, "no forcing pass yet");
    if ((long long)h->n_markers > (long long)kNoAllocChunk * kNoAllocMaxBlocks)
        return fail(h, TDLB_EINVAL, "marker list longer than the 1048576 markers tdlb_impeller_load_noalloc supports");
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, TDLB_ECUDA, "cudaSetDevice failed");
    if (tdlb_rt::join_side(h) != cudaSuccess) return fail(h, TDLB_ECUDA, "join of the split-step stream failed");
    double* partial = nullptr;
    if (partials_address(h->device, &partial) != cudaSuccess)
        return fail(h, TDLB_ECUDA, "cudaGetSymbolAddress of the no-allocation scratch failed");
    const int n = h->n_markers;
    const int blocks = n > 0 ? (n + kNoAllocChunk - 1) / kNoAllocChunk : 1;
    k_marker_load_chunks<<<blocks, 256, 0, h->stream>>>(h->d_sums, h->d_sched, h->d_markers, n, h->impeller_begin,
                                                        h->last_beta, h->rot_ci, h->rot_ck, partial);
    k_marker_load_chunks_final<<<1, 32, 0, h->stream>>>(partial, blocks, d_out5);
    if (cudaGetLastError() != cudaSuccess) return fail(h, TDLB_ECUDA, "kernel launch failed");
    return TDLB_OK;
}
