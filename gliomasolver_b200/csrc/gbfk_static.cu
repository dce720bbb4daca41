// gbfk_rd_step_static: one fused RD step on a uniform periodic grid that
// allocates no device memory.
//
// Who needs it: a caller whose device memory is owned by another allocator
// (a framework that reserved the GPU's memory up front and hands out
// sub-buffers), or a time loop that must not pay cudaMalloc's device-wide
// synchronisation, cannot let the library allocate its per-call scratch.
// This variant keeps that scratch -- the harmonic-mean face coefficients, the
// per-cell meta words, the block types and the neighbour table of the fused
// step -- in one file-scope device array of fixed size instead of memory from
// cudaMalloc.  The caller passes device pointers to the inputs and the output.
//
// Limits and sharing:
//  - at most GBFK_STATIC_MAX_BLOCKS (512) blocks of 8^3 cells, i.e. up to a
//    64^3 grid; larger grids are rejected with GBFK_E_TOO_LARGE;
//  - the array costs about 7.3 MiB on every GPU that loads the library and is
//    held until the process exits;
//  - every call on a device uses the same array, and the array keeps the last
//    call's contents; each call rewrites all of it before reading it, so
//    nothing carries over from one call to the next, but two calls whose work
//    overlaps on the GPU (different streams or threads, same device) race on
//    the array and give wrong results.  Serialise them.
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.  The address is kept with the ID of the
//    device's context and looked up again if the context changed (after a
//    cudaDeviceReset, say).
//  - no NaN check: the step kernel's NaN flag lives in the shared array and
//    is not reported; a step that produces NaN or Inf returns GBFK_OK.
//  - the caller's current device is restored before returning; an error that
//    the caller's earlier work left pending is returned as GBFK_E_CUDA and
//    not cleared.
#include "gbfk.h"
#include "gbfk_kernels.cuh"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

namespace gbfk {

constexpr int kStaticMaxBlocks = GBFK_STATIC_MAX_BLOCKS;
// section sizes for the widest Real (double), each a multiple of 256 bytes
constexpr size_t kStaticH = (size_t)kStaticMaxBlocks * kFacesPerBlock * sizeof(double);
constexpr size_t kStaticMeta = (size_t)kStaticMaxBlocks * kBS3 * sizeof(unsigned short);
constexpr size_t kStaticBtype = 512;
constexpr size_t kStaticNbr = (size_t)kStaticMaxBlocks * 6 * sizeof(int);
constexpr size_t kStaticIh2 = (size_t)kStaticMaxBlocks * sizeof(double);
constexpr size_t kStaticSlot = (size_t)kStaticMaxBlocks * sizeof(int);
constexpr size_t kStaticFlag = 256;
constexpr size_t kStaticBytes =
    kStaticH + kStaticMeta + kStaticBtype + kStaticNbr + kStaticIh2 + kStaticSlot + kStaticFlag;
static_assert(kStaticBtype >= (size_t)kStaticMaxBlocks, "block types section too small");

// The scratch itself.  In host code this name is only a host-side stand-in
// for the device array, not a device address: the address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

namespace {

std::mutex g_static_mutex;
unsigned char *g_static_ptr[64] = {};
unsigned long long g_static_ctx[64] = {};

// Unique ID of the current context (cuCtxGetId through the runtime's driver
// entry points); 0 if it cannot be had.
unsigned long long current_context_id()
{
    typedef CUresult (*GetCurrent)(CUcontext *);
    typedef CUresult (*GetId)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)p;
        p = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)p;
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
    return 0;
}

// Neighbour table, slot table and 1/(h*h) of a uniform periodic bpd^3 grid,
// written on the device (block b = bx + bpd*(by + bpd*bz) lives in slot b).
__global__ void static_topology_kernel(int bpd, double ih2, int *nbr, double *ih2blk, int *slot)
{
    const int nb = bpd * bpd * bpd;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int bx = b % bpd, by = (b / bpd) % bpd, bz = b / (bpd * bpd);
        auto id = [&](int x, int y, int z) {
            x = (x + bpd) % bpd;
            y = (y + bpd) % bpd;
            z = (z + bpd) % bpd;
            return x + bpd * (y + bpd * z);
        };
        nbr[b * 6 + 0] = id(bx - 1, by, bz);
        nbr[b * 6 + 1] = id(bx + 1, by, bz);
        nbr[b * 6 + 2] = id(bx, by - 1, bz);
        nbr[b * 6 + 3] = id(bx, by + 1, bz);
        nbr[b * 6 + 4] = id(bx, by, bz - 1);
        nbr[b * 6 + 5] = id(bx, by, bz + 1);
        ih2blk[b] = ih2;
        slot[b] = b;
    }
}

// The array's device address on `device` (current): looked up once per device
// and context.
int static_scratch(int device, unsigned char **out)
{
    std::lock_guard<std::mutex> lk(g_static_mutex);
    if (device < 0 || device >= 64) return GBFK_E_INVALID;
    const unsigned long long ctx = current_context_id();
    if (!g_static_ptr[device] || ctx != g_static_ctx[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) return GBFK_E_CUDA;
        g_static_ptr[device] = (unsigned char *)p;
        g_static_ctx[device] = ctx;
    }
    *out = g_static_ptr[device];
    return GBFK_OK;
}

template <typename Real>
int static_step(unsigned char *scratch, int bpd, const void *pw, const void *pg, const void *phi_in, void *phi_out,
                double Dw, double Dg, double rho, double dt, cudaStream_t s)
{
    Real *H = (Real *)scratch;
    unsigned short *meta = (unsigned short *)(scratch + kStaticH);
    unsigned char *btype = scratch + kStaticH + kStaticMeta;
    int *nbr = (int *)(scratch + kStaticH + kStaticMeta + kStaticBtype);
    double *ih2 = (double *)(scratch + kStaticH + kStaticMeta + kStaticBtype + kStaticNbr);
    int *slot = (int *)(scratch + kStaticH + kStaticMeta + kStaticBtype + kStaticNbr + kStaticIh2);
    unsigned *flag =
        (unsigned *)(scratch + kStaticH + kStaticMeta + kStaticBtype + kStaticNbr + kStaticIh2 + kStaticSlot);

    const int nb = bpd * bpd * bpd;
    const double h = (double)(Real)(1.0 / (8.0 * bpd));
    static_topology_kernel<<<(nb + 127) / 128, 128, 0, s>>>(bpd, 1. / (h * h), nbr, ih2, slot);
    if (cudaGetLastError() != cudaSuccess) return GBFK_E_CUDA;
    if (cudaMemsetAsync(flag, 0, sizeof(unsigned), s) != cudaSuccess) return GBFK_E_CUDA;

    PoolView<Real> v;
    v.slot = slot;
    v.nbr = nbr;
    v.hblk = nullptr;
    v.gpw = v.gpg = v.gphi = nullptr;
    v.pw = (const Real *)pw;
    v.pg = (const Real *)pg;
    v.btype = btype;
    v.nblocks = nb;
    v.identity_slots = 1;
    v.log2_bpd = -1;
    if (launch_faces<Real>(v, (Real)Dw, (Real)Dg, H, meta, btype, s) != cudaSuccess) return GBFK_E_CUDA;
    if (launch_rd_step<Real>(v, H, meta, ih2, (const Real *)phi_in, (Real *)phi_out, nullptr, (Real)rho, dt, flag,
                             s) != cudaSuccess)
        return GBFK_E_CUDA;
    return GBFK_OK;
}

// Restores the caller's current device when the entry point returns.
struct DeviceGuard {
    int saved = -1;
    DeviceGuard() { if (cudaGetDevice(&saved) != cudaSuccess) saved = -1; }
    ~DeviceGuard() { if (saved >= 0) cudaSetDevice(saved); }
};

}  // namespace
}  // namespace gbfk

extern "C" int gbfk_rd_step_static(int precision, int bpd, const void *pw, const void *pg, const void *phi_in,
                                   void *phi_out, double Dw, double Dg, double rho, double dt, void *stream,
                                   int device)
{
    using namespace gbfk;
    if (precision != GBFK_F64 && precision != GBFK_F32) return GBFK_E_INVALID;
    if (bpd <= 0) return GBFK_E_INVALID;
    if ((long long)bpd * bpd * bpd > kStaticMaxBlocks) return GBFK_E_TOO_LARGE;
    if (!pw || !pg || !phi_in || !phi_out) return GBFK_E_INVALID;
    // phi_out must not overlap phi_in anywhere: the step reads neighbours'
    // halos from phi_in while other CTAs write phi_out
    const uintptr_t bytes = (uintptr_t)bpd * bpd * bpd * 512 * (precision == GBFK_F64 ? 8 : 4);
    const uintptr_t in0 = (uintptr_t)phi_in, out0 = (uintptr_t)phi_out;
    if (in0 < out0 + bytes && out0 < in0 + bytes) return GBFK_E_INVALID;
    DeviceGuard guard;
    if (cudaSetDevice(device) != cudaSuccess) return GBFK_E_CUDA;
    // an error left pending by the caller's own earlier work is reported and
    // left in place, so that the launch checks below see only this call's
    if (cudaPeekAtLastError() != cudaSuccess) return GBFK_E_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        // the stream must belong to `device`
        int sdev = -1;
        if (cudaStreamGetDevice(s, &sdev) != cudaSuccess || sdev != device) return GBFK_E_INVALID;
    }
    unsigned char *scratch = nullptr;
    const int rc = static_scratch(device, &scratch);
    if (rc != GBFK_OK) return rc;
    return precision == GBFK_F64 ? static_step<double>(scratch, bpd, pw, pg, phi_in, phi_out, Dw, Dg, rho, dt, s)
                                 : static_step<float>(scratch, bpd, pw, pg, phi_in, phi_out, Dw, Dg, rho, dt, s);
}
