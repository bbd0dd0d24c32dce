// mb_noalloc.cu -- Compute_dt of one block with no device allocation (mb_dt_block_noalloc).
//
// Some callers of this library cannot allocate device memory at the moment they need a time step:
//  - a Fortran host whose device memory is owned by the OpenACC runtime (the reference's present table),
//    through a thin ISO_C_BINDING shim that must not create device buffers behind that runtime's back;
//  - a serving loop that has already admitted cases up to its HBM budget;
//  - code that must not stall the device: cudaMalloc / cudaFree synchronise, and they are not allowed
//    while a stream is being captured into a CUDA graph.
// mb_dt needs a context from mb_init, which allocates; this entry point takes everything as caller-owned
// device pointers and keeps its only scratch -- the per-CTA partial minima of the reduction -- in the
// file-scope array below, which every GPU that loads the library holds until the process exits.
//
// Reduction: pass 1 writes one partial minimum per CTA into the array (every slot that pass 2 reads is
// written by the same call first, so nothing needs clearing); pass 2, one CTA, folds the slots in a
// fixed order and writes min(1e5, minimum) to the caller's output, as Compute_dt's dtglobal
// (numerics/time/Mod_dt.f90:15-106; Mod_Explicit.f90:122). The local dt of a cell is cell_dt of
// mb_engine.cuh, the FP64 arithmetic of mb_dt's parity form, whatever the scheme's precision (the mixed form's mb_dt
// takes it in FP32), and the cfl-rise ramp is not applied: the caller multiplies by iter / cfl_rise during the ramp.
// Built with --fmad=false like the FP64 form.
#include <cstdio>
#include <cstring>
#include "../../include/mose_b200.h"
#include "mb_engine.cuh"

namespace {

constexpr int kMaxPartials = 65536;  // 512 KB of partial minima: the stated maximum of this entry point
constexpr int kTY = 8;               // tile: 32 (i) x 8 (j) cells, a chunk of k planes per CTA
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partials[kMaxPartials];

// device address of g_partials per device (looked up once per device, with that device current)
double* g_partials_addr[kMaxDevices] = {nullptr};

__global__ void __launch_bounds__(32 * kTY) k_dt_partials(mb::Params p, mb::DBlk b, const double* __restrict__ P,
                                                         int ti, int tj, int kc, double* __restrict__ partials) {
  __shared__ double sred[32];
  const int t = blockIdx.x;
  const int it = t % ti, jt = (t / ti) % tj, kt = t / (ti * tj);
  const int i = 1 + 32 * it + (threadIdx.x & 31), j = 1 + kTY * jt + (threadIdx.x >> 5);
  const int k0 = 1 + kc * kt, k1 = min(k0 + kc, b.n3 + 1);
  double v = 1e300;
  if (i <= b.n1 && j <= b.n2) {
    for (int k = k0; k < k1; ++k) {
      const long long r = mb::row(b, i, j, k);
      double pl[MB_NP];
      for (int s = 0; s < MB_NP; ++s) pl[s] = P[r + s * p.nc];
      v = mb::mn(v, mb::cell_dt(p, b, r - b.boff, pl));
    }
  }
  const unsigned full = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) v = mb::mn(v, __shfl_xor_sync(full, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sred[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < kTY) ? sred[lane] : 1e300;
    for (int o = 16; o > 0; o >>= 1) v = mb::mn(v, __shfl_xor_sync(full, v, o));
    if (lane == 0) partials[t] = v;
  }
}

__global__ void __launch_bounds__(1024) k_dt_fold(const double* __restrict__ partials, int n, double* dt_out) {
  __shared__ double sred[32];
  double v = 1e300;
  for (int q = threadIdx.x; q < n; q += blockDim.x) v = mb::mn(v, partials[q]);
  const unsigned full = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) v = mb::mn(v, __shfl_xor_sync(full, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sred[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sred[lane] : 1e300;
    for (int o = 16; o > 0; o >>= 1) v = mb::mn(v, __shfl_xor_sync(full, v, o));
    if (lane == 0) *dt_out = mb::mn(v, 1e5);
  }
}

}  // namespace

// the tile decomposition of a block: 32 x 8 cells per (i, j) tile; the k chunk starts at 16 planes and doubles until
// the partial minima (one per tile) fit the static array. Tile t covers i-tile t % ti, j-tile (t / ti) % tj and the
// planes 1 + kc * (t / (ti * tj)) .. min(that + kc, n3 + 1) - 1.
static int dt_tiles(const int32_t n[3], long long* ti, long long* tj, long long* kc, long long* ntiles) {
  if (!n || n[0] < 1 || n[1] < 1 || n[2] < 1) return MB_E_ARG;
  *ti = (n[0] + 31) / 32;
  *tj = (n[1] + kTY - 1) / kTY;
  if (*ti * *tj > kMaxPartials) return MB_E_ARG;
  *kc = 16;
  while (*ti * *tj * ((n[2] + *kc - 1) / *kc) > kMaxPartials) *kc *= 2;
  *ntiles = *ti * *tj * ((n[2] + *kc - 1) / *kc);
  return MB_OK;
}

extern "C" int mb_dt_block_noalloc_tiles(const int32_t n[3], int32_t* kc, int32_t* ntiles) {
  long long ti, tj, k, nt;
  const int rc = dt_tiles(n, &ti, &tj, &k, &nt);
  if (rc != MB_OK) return rc;
  if (kc) *kc = (int32_t)k;
  if (ntiles) *ntiles = (int32_t)nt;
  return MB_OK;
}

extern "C" int mb_dt_block_noalloc(const double* P, int64_t ncell_total, int64_t boff, const int32_t n[3],
                                   const double* dl, const double* m, const double* cp, const double* mu,
                                   const double* k, int32_t tmin, int32_t tmax, double wm, const mb_scheme* sc,
                                   double* dt_out, void* stream) {
  if (!P || !n || !dl || !m || !cp || !mu || !k || !sc || !dt_out) return MB_E_ARG;
  if (n[0] < 1 || n[1] < 1 || n[2] < 1 || tmax - tmin < 2 || ncell_total < 1 || boff < 0) return MB_E_ARG;
  if (sc->ndir < 1 || sc->ndir > 3) return MB_E_ARG;
  // preconditioning takes its steps from the Ur field of the context (pseudo-acoustic speed): not served here
  if (sc->intvar == 2) {
    fprintf(stderr, "[mose_b200] mb_dt_block_noalloc: integration-variables = prec needs the Ur field of a context "
                    "(mb_dt)\n");
    return MB_E_UNSUPPORTED;
  }
  const long long pi = n[0] + 2 * MB_GC, pj = n[1] + 2 * MB_GC, pk = n[2] + 2 * MB_GC;
  if (boff + pi * pj * pk > ncell_total) return MB_E_ARG;
  long long ti, tj, kc, nt;
  if (dt_tiles(n, &ti, &tj, &kc, &nt) != MB_OK) {
    fprintf(stderr, "[mose_b200] mb_dt_block_noalloc: a %d x %d plane needs %lld partial minima, more than the "
                    "%d of its static scratch\n", n[0], n[1], ti * tj, kMaxPartials);
    return MB_E_ARG;
  }
  const int ntiles = (int)nt;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MB_E_CUDA;
  if (!g_partials_addr[dev]) {
    // set-up, once per device: the host name g_partials is only a stand-in for the device array. The look-up may
    // not run inside a stream capture (it would fail or invalidate the capture), so a first call made while the
    // stream is capturing is refused with a message
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      fprintf(stderr, "[mose_b200] mb_dt_block_noalloc: the first call on a device sets up the device address of its "
                      "scratch and cannot run while the stream is being captured; make one call before the capture\n");
      return MB_E_ARG;
    }
    void* a = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&a, g_partials);
    if (e != cudaSuccess || !a) {
      fprintf(stderr, "[mose_b200] mb_dt_block_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return MB_E_CUDA;
    }
    g_partials_addr[dev] = (double*)a;
  }
  mb::Params p;
  memset(&p, 0, sizeof(p));
  p.cp = cp - tmin;
  p.mu = mu - tmin;
  p.k = k - tmin;
  p.h = nullptr;
  p.nc = ncell_total;
  p.tmin = tmin;
  p.tmax = tmax;
  p.wm = wm;
  p.ri = mb::RUNIV / wm;
  p.visc = sc->visc ? 1 : 0;
  p.ndir = sc->ndir;
  p.dt_additive = sc->dt_additive;
  p.cfl = sc->cfl;
  p.vnn = sc->vnn;
  p.prandtl = sc->prandtl;
  mb::DBlk b;
  memset(&b, 0, sizeof(b));
  b.n1 = n[0]; b.n2 = n[1]; b.n3 = n[2];
  b.pi = (int)pi; b.pj = (int)pj;
  b.grp = 0; b.ndir = sc->ndir;
  b.boff = boff;
  b.dl = dl;
  b.m = m;
  for (int f = 0; f < 6; ++f) b.rmap[f] = -1;
  k_dt_partials<<<ntiles, 32 * kTY, 0, s>>>(p, b, P, (int)ti, (int)tj, (int)kc, g_partials_addr[dev]);
  k_dt_fold<<<1, 1024, 0, s>>>(g_partials_addr[dev], ntiles, dt_out);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_E_CUDA;
}
