// Summation density with no device allocation (simp_gpu_sum_density_noalloc).
//
// Who needs it: callers that must not call cudaMalloc.  A host whose device
// memory belongs to another runtime (CUDA Fortran or OpenACC device arrays,
// a framework's caching allocator) cannot let a library allocate behind its
// back, and a loop that may not stall cannot afford cudaMalloc, which can
// synchronise the whole device.  Such a caller owns its input and output
// buffers already; this entry point only needs working memory for its cell
// list, and takes it from one fixed array compiled into the library.
//
// The working memory is the file-scope array g_noalloc_scratch below
// (kNoAllocScratchBytes, about 7 MB).  Every GPU that loads the library
// holds it until the process exits.  Host code cannot use the array's name as
// a device address, so the first call on each device looks the address up
// with cudaGetSymbolAddress (with that device current) and passes it to the
// kernels; the address is looked up again when a different CUDA context is
// current on that device (after cudaDeviceReset, or a context the caller
// made itself).  The first call on a device (and the first after such a
// change) should come before any stream capture.  All calls share the array
// and it keeps the last call's contents: everything that must start at zero
// is cleared at the start of each call, and calls that overlap on the GPU
// (different streams, or different host threads on one device) race on it
// and must be serialised by the caller.
//
// Order within a cell: particles are put in cell order by a stable radix
// sort of their cell keys (the input is in particle-index order, so each
// cell lists its particles by increasing index), which makes every call's
// summation order, and so its bits, reproducible.  The sort works in the
// same fixed array (CUB's device radix sort given that storage; it
// allocates nothing itself).
#include <cstdint>
#include <mutex>

#include <cub/device/device_radix_sort.cuh>

#include "ctx.h"
#include "neighbors.cuh"

namespace simp {
namespace noalloc {

constexpr int kMaxN = SIMP_NOALLOC_MAX_PARTICLES;
constexpr int kMaxCells = 2 * SIMP_NOALLOC_MAX_PARTICLES;
constexpr int kKeyBits = 17;                 // cell keys < kMaxCells = 2^17
static_assert(kMaxCells <= (1 << kKeyBits), "cell keys exceed the sorted bits");
constexpr int kB = 128;
// working storage handed to the radix sort (checked against its own
// request at each call)
constexpr size_t kSortTempBytes = size_t(2) << 20;

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

struct Header {
    Grid grid;
    Scalars sc;                          // hmin, hmax, bs for the bucket rule
    unsigned long long xmin, xmax, ymin, ymax, hmin, hmax;  // order-preserving bits
};

constexpr size_t kOffHeader = 0;
constexpr size_t kOffCnt = align256(kOffHeader + sizeof(Header));
constexpr size_t kOffStart = align256(kOffCnt + sizeof(int) * (kMaxCells + 1));
constexpr size_t kOffScan = align256(kOffStart + sizeof(int) * (kMaxCells + 1));
constexpr size_t kOffKey = align256(kOffScan + sizeof(int) * ((kMaxCells + 1) / 1024 + 2));
constexpr size_t kOffKeySorted = align256(kOffKey + sizeof(int) * kMaxN);
constexpr size_t kOffIota = align256(kOffKeySorted + sizeof(int) * kMaxN);
constexpr size_t kOffPerm = align256(kOffIota + sizeof(int) * kMaxN);
constexpr size_t kOffX = align256(kOffPerm + sizeof(int) * kMaxN);
constexpr size_t kOffY = kOffX + sizeof(double) * kMaxN;
constexpr size_t kOffHs = kOffY + sizeof(double) * kMaxN;
constexpr size_t kOffM = kOffHs + sizeof(double) * kMaxN;
constexpr size_t kOffRho = kOffM + sizeof(double) * kMaxN;
constexpr size_t kOffSort = align256(kOffRho + sizeof(double) * kMaxN);
constexpr size_t kNoAllocScratchBytes = align256(kOffSort + kSortTempBytes);

static_assert(sizeof(int) * ((kMaxCells + 1) / 1024 + 2) >= sizeof(int) * ((kMaxCells + 1023) / 1024 + 1),
              "scan scratch too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

template <class T>
__host__ __device__ __forceinline__ T *at(unsigned char *base, size_t off) {
    return reinterpret_cast<T *>(base + off);
}

// order-preserving map of a double onto unsigned 64-bit integers
__device__ __forceinline__ unsigned long long ord(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord(unsigned long long u) {
    const unsigned long long b = (u >> 63) ? (u ^ 0x8000000000000000ull) : ~u;
    return __longlong_as_double((long long)b);
}

__global__ void k_clear(unsigned char *base) {
    int *cnt = at<int>(base, kOffCnt);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= kMaxCells; c += gridDim.x * blockDim.x) cnt[c] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Header *h = at<Header>(base, kOffHeader);
        h->xmin = h->ymin = h->hmin = ~0ull;
        h->xmax = h->ymax = h->hmax = 0ull;
    }
}

// Extents: each block folds its particles' six bounds with warp shuffles and
// one shared-memory pass, then issues one atomic per bound.
__global__ void __launch_bounds__(kB) k_bounds(unsigned char *base, int n, const double *__restrict__ x,
                                               const double *__restrict__ hs) {
    __shared__ unsigned long long part[kB / 32][6];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    // (lanes past n carry neutral values)
    unsigned long long v[6] = {~0ull, 0ull, ~0ull, 0ull, ~0ull, 0ull};   // min, max of x, y, hsml
    if (i < n) {
        const unsigned long long ox = ord(x[2 * i]), oy = ord(x[2 * i + 1]), oh = ord(hs[i]);
        v[0] = v[1] = ox;
        v[2] = v[3] = oy;
        v[4] = v[5] = oh;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, v[q], o);
            v[q] = (q & 1) ? (t > v[q] ? t : v[q]) : (t < v[q] ? t : v[q]);
        }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 6; ++q) part[w][q] = v[q];
    __syncthreads();
    const int q = threadIdx.x;
    if (q < 6) {
        unsigned long long r = part[0][q];
        for (int k = 1; k < kB / 32; ++k) r = (q & 1) ? (part[k][q] > r ? part[k][q] : r) : (part[k][q] < r ? part[k][q] : r);
        Header *h = at<Header>(base, kOffHeader);
        switch (q) {
            case 0: atomicMin(&h->xmin, r); break;
            case 1: atomicMax(&h->xmax, r); break;
            case 2: atomicMin(&h->ymin, r); break;
            case 3: atomicMax(&h->ymax, r); break;
            case 4: atomicMin(&h->hmin, r); break;
            default: atomicMax(&h->hmax, r); break;
        }
    }
}

// Grid over the particles' extent with side >= max(hsml); at most kMaxCells.
__global__ void k_grid(unsigned char *base) {
    Header *h = at<Header>(base, kOffHeader);
    const double xmin = unord(h->xmin), xmax = unord(h->xmax);
    const double ymin = unord(h->ymin), ymax = unord(h->ymax);
    const double hmin = unord(h->hmin), hmax = unord(h->hmax);
    double cs = hmax * (1.0 + 1e-6);
    // invalid input (hsml <= 0, non-finite positions): one cell, finite size;
    // the results are then meaningless but every loop stays bounded
    const bool ok = cs > 0.0 && isfinite(cs) && isfinite(xmax - xmin) && isfinite(ymax - ymin);
    if (!ok) cs = 1.0;
    const double w = ok ? (xmax - xmin) + 2.0 * cs : 1.0, hh = ok ? (ymax - ymin) + 2.0 * cs : 1.0;
    for (int it = 0; it < 400 && ceil(w / cs) * ceil(hh / cs) > (double)kMaxCells; ++it) cs *= 1.25;
    Grid g;
    g.x0 = ok ? xmin - cs : 0.0;
    g.y0 = ok ? ymin - cs : 0.0;
    g.cs = cs;
    g.inv_cs = 1.0 / cs;
    g.ncx = min(kMaxCells, max(1, (int)ceil(w / cs)));
    g.ncy = min(kMaxCells / g.ncx, max(1, (int)ceil(hh / cs)));
    g.base = 0;
    g.cell_start = at<int>(base, kOffStart);
    h->grid = g;
    Scalars s{};
    s.hmin = hmin;
    s.hmax = hmax;
    s.bs = 2.0 * hmin;
    s.dmax2_bits = 0ull;
    h->sc = s;
}

// Cell key of each particle (the sort's keys) and its index (the sort's
// values), plus the per-cell counts whose scan gives the cell starts.
__global__ void k_keys(unsigned char *base, int n, const double *__restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Grid g = at<Header>(base, kOffHeader)->grid;
    const int cx = clampi((int)floor((x[2 * i] - g.x0) * g.inv_cs), 0, g.ncx - 1);
    const int cy = clampi((int)floor((x[2 * i + 1] - g.y0) * g.inv_cs), 0, g.ncy - 1);
    const int k = cy * g.ncx + cx;
    at<int>(base, kOffKey)[i] = k;
    at<int>(base, kOffIota)[i] = i;
    atomicAdd(&at<int>(base, kOffCnt)[k], 1);
}

// Sorted copy of the particles; keys[k] is the cell of sorted position k.
__global__ void k_gather(unsigned char *base, int n, const double *__restrict__ x,
                         const double *__restrict__ hs, const double *__restrict__ m,
                         const double *__restrict__ rho) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = at<int>(base, kOffPerm)[k];
    at<double>(base, kOffX)[k] = x[2 * o];
    at<double>(base, kOffY)[k] = x[2 * o + 1];
    at<double>(base, kOffHs)[k] = hs[o];
    at<double>(base, kOffM)[k] = m[o];
    at<double>(base, kOffRho)[k] = rho[o];
}

// density.f90:74-98 on the sorted copy; kernel_zero from the particle's hsml.
__global__ void __launch_bounds__(kB) k_density(unsigned char *base, int n, Phys P, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Header *hd = at<Header>(base, kOffHeader);
    const Grid g = hd->grid;
    const double *X = at<double>(base, kOffX), *Y = at<double>(base, kOffY);
    const double *HS = at<double>(base, kOffHs), *M = at<double>(base, kOffM);
    const double *RHO = at<double>(base, kOffRho);
    const double xi = X[i], yi = Y[i], hi = HS[i];
    const BinRule br = make_bin_rule(hd->sc.bs, xi, yi, hd->sc.hmax);
    const double k0 = kernel_zero(P, hi);
    const double mi = M[i];
    double num = k0 * mi, den = k0 * mi / RHO[i];
    for_each_pair(X, Y, HS, g, i, at<int>(base, kOffKeySorted)[i], 1, br, xi, yi, hi,
                  [&](int j, double, double, double r, double mh) {
                      double w, gf;
                      pair_kernel<true>(P, r, mh, &w, &gf);
                      const double mw = M[j] * w;
                      den += mw / RHO[j];
                      num += mw;
                  });
    out[at<int>(base, kOffPerm)[i]] = num / den;
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

// The stable radix sort of the cell keys, in the fixed array's storage.  The
// sort first states how much storage it needs for n keys (a host-side
// query that launches nothing); more than the set-aside is an error.
cudaError_t sort_keys(unsigned char *base, int n, cudaStream_t s) {
    const int *kin = at<int>(base, kOffKey);
    int *kout = at<int>(base, kOffKeySorted);
    const int *vin = at<int>(base, kOffIota);
    int *vout = at<int>(base, kOffPerm);
    size_t need = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, need, kin, kout, vin, vout, n, 0, kKeyBits, s);
    if (e != cudaSuccess) return e;
    if (need > kSortTempBytes) return cudaErrorMemoryAllocation;
    size_t bytes = kSortTempBytes;
    return cub::DeviceRadixSort::SortPairs(base + kOffSort, bytes, kin, kout, vin, vout, n, 0, kKeyBits, s);
}

// Device address of the scratch array, looked up once per device and again
// whenever another CUDA context is current on it.
constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char *g_addr[kMaxDevices] = {};
void *g_ctx[kMaxDevices] = {};

// The current driver context, read through the runtime's driver entry point
// (the library links only the runtime).
using CtxGetCurrent = int (*)(void **);
CtxGetCurrent ctx_get_current() {
    static CtxGetCurrent fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<CtxGetCurrent>(p);
    }();
    return fn;
}

cudaError_t scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    void *ctx = nullptr;
    if (CtxGetCurrent f = ctx_get_current()) f(&ctx);
    std::lock_guard<std::mutex> lk(g_lock);
    if (!g_addr[dev] || g_ctx[dev] != ctx) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<unsigned char *>(p);
        // (the runtime has made its primary context current by now)
        ctx = nullptr;
        if (CtxGetCurrent f = ctx_get_current()) f(&ctx);
        g_ctx[dev] = ctx;
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

// A buffer the kernels may read or write: device memory of the current
// device, or managed memory.  A host array (pageable or pinned) is refused.
bool device_buffer(const void *p, int dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();   // (clears the error this query may record)
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace noalloc
}  // namespace simp

extern "C" int32_t simp_gpu_sum_density_noalloc(const double *x, const double *hsml, const double *mass,
                                                const double *rho, int32_t n, int32_t skf,
                                                double *rho_out, void *stream) {
    using namespace simp;
    using namespace simp::noalloc;
    if (n < 1 || n > kMaxN || !x || !hsml || !mass || !rho || !rho_out) return SIMP_ERR_BADARG;
    if (!skf_known(skf)) return SIMP_ERR_BADARG;
    // an error left by earlier work on this thread is the caller's: report
    // it without launching, and leave it in place
    if (cudaPeekAtLastError() != cudaSuccess) return SIMP_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SIMP_ERR_CUDA;
    const void *bufs[5] = {x, hsml, mass, rho, rho_out};
    for (const void *p : bufs)
        if (!device_buffer(p, dev)) return SIMP_ERR_BADARG;
    unsigned char *base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return SIMP_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Phys P{};
    P.skf = skf;
    P.scale_h = scale_h_of(skf);
    k_clear<<<nblk(kMaxCells + 1, 256), 256, 0, s>>>(base);
    k_bounds<<<nblk(n, kB), kB, 0, s>>>(base, n, x, hsml);
    k_grid<<<1, 1, 0, s>>>(base);
    k_keys<<<nblk(n, kB), kB, 0, s>>>(base, n, x);
    launch_scan_i32(at<int>(base, kOffCnt), at<int>(base, kOffStart), kMaxCells, base + kOffScan, s);
    if (sort_keys(base, n, s) != cudaSuccess) return SIMP_ERR_CUDA;
    k_gather<<<nblk(n, kB), kB, 0, s>>>(base, n, x, hsml, mass, rho);
    k_density<<<nblk(n, kB), kB, 0, s>>>(base, n, P, rho_out);
    return cudaGetLastError() == cudaSuccess ? SIMP_OK : SIMP_ERR_CUDA;
}
