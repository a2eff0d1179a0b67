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
// (kNoAllocScratchBytes, about 5 MB).  Every GPU that loads the library
// holds it until the process exits.  Host code cannot use the array's name as
// a device address, so the first call on each device looks the address up
// with cudaGetSymbolAddress (with that device current) and passes it to the
// kernels.  That first call should come before any stream capture.  All calls
// share the array and it keeps the last call's contents: everything that
// must start at zero is cleared at the start of each call, and calls that
// overlap on the GPU (different streams, or different host threads on one
// device) race on it and must be serialised by the caller.
#include <cstdint>
#include <mutex>

#include "ctx.h"
#include "neighbors.cuh"

namespace simp {
namespace noalloc {

constexpr int kMaxN = SIMP_NOALLOC_MAX_PARTICLES;
constexpr int kMaxCells = 2 * SIMP_NOALLOC_MAX_PARTICLES;
constexpr int kB = 128;

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
constexpr size_t kOffPerm = align256(kOffKey + sizeof(int) * kMaxN);
constexpr size_t kOffScell = align256(kOffPerm + sizeof(int) * kMaxN);
constexpr size_t kOffX = align256(kOffScell + sizeof(int) * kMaxN);
constexpr size_t kOffY = kOffX + sizeof(double) * kMaxN;
constexpr size_t kOffHs = kOffY + sizeof(double) * kMaxN;
constexpr size_t kOffM = kOffHs + sizeof(double) * kMaxN;
constexpr size_t kOffRho = kOffM + sizeof(double) * kMaxN;
constexpr size_t kNoAllocScratchBytes = align256(kOffRho + sizeof(double) * kMaxN);

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

__global__ void k_bounds(unsigned char *base, int n, const double *__restrict__ x,
                         const double *__restrict__ hs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Header *h = at<Header>(base, kOffHeader);
    atomicMin(&h->xmin, ord(x[2 * i]));
    atomicMax(&h->xmax, ord(x[2 * i]));
    atomicMin(&h->ymin, ord(x[2 * i + 1]));
    atomicMax(&h->ymax, ord(x[2 * i + 1]));
    atomicMin(&h->hmin, ord(hs[i]));
    atomicMax(&h->hmax, ord(hs[i]));
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

__global__ void k_keys(unsigned char *base, int n, const double *__restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Grid g = at<Header>(base, kOffHeader)->grid;
    const int cx = clampi((int)floor((x[2 * i] - g.x0) * g.inv_cs), 0, g.ncx - 1);
    const int cy = clampi((int)floor((x[2 * i + 1] - g.y0) * g.inv_cs), 0, g.ncy - 1);
    const int k = cy * g.ncx + cx;
    at<int>(base, kOffKey)[i] = k;
    atomicAdd(&at<int>(base, kOffCnt)[k], 1);
}

__global__ void k_scatter(unsigned char *base, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = at<int>(base, kOffKey)[i];
    const int slot = atomicSub(&at<int>(base, kOffCnt)[k], 1) - 1;
    at<int>(base, kOffPerm)[at<int>(base, kOffStart)[k] + slot] = i;
}

// deterministic order inside a cell: ascending particle index
__global__ void k_cell_sort(unsigned char *base) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Grid g = at<Header>(base, kOffHeader)->grid;
    if (c >= g.ncx * g.ncy) return;
    const int *start = at<int>(base, kOffStart);
    int *perm = at<int>(base, kOffPerm);
    const int a = start[c], b = start[c + 1];
    for (int k = a + 1; k < b; ++k) {
        const int v = perm[k];
        int j = k - 1;
        while (j >= a && perm[j] > v) { perm[j + 1] = perm[j]; --j; }
        perm[j + 1] = v;
    }
}

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
    at<int>(base, kOffScell)[k] = at<int>(base, kOffKey)[o];
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
    for_each_pair(X, Y, HS, g, i, at<int>(base, kOffScell)[i], 1, br, xi, yi, hi,
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

// Device address of the scratch array, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char *g_addr[kMaxDevices] = {};

cudaError_t scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_lock);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
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
    k_scatter<<<nblk(n, kB), kB, 0, s>>>(base, n);
    k_cell_sort<<<nblk(kMaxCells, kB), kB, 0, s>>>(base);
    k_gather<<<nblk(n, kB), kB, 0, s>>>(base, n, x, hsml, mass, rho);
    k_density<<<nblk(n, kB), kB, 0, s>>>(base, n, P, rho_out);
    return cudaGetLastError() == cudaSuccess ? SIMP_OK : SIMP_ERR_CUDA;
}
