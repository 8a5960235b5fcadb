// margins_static.cu -- clgpu_margins_static: the margins computation of
// clgpu_margins (cones_api.cu) for callers that must not allocate device
// memory and hold no cone handle.
//
// The cone layout and the per-cone temporaries live in one file-scope
// __device__ array of fixed size instead of buffers allocated by
// clgpu_cones_create.  The kernels are the same launcher, cones_margins
// (cones.cu); only where their scratch lives differs.
//
//   * The first call on each device resolves the array's address with
//     cudaGetSymbolAddress while that device is current; make that first call
//     before any stream capture begins.
//   * Nothing here calls cudaMalloc, cudaFree or an allocating library
//     routine.  Sizes above CLGPU_MARGINS_STATIC_MAX_CONES second-order plus
//     PSD cones return CLGPU_ERR_STATIC_TOO_LARGE.
//   * Every scratch word a call reads is written earlier in the same call
//     (layout by the upload, per-cone temporaries by the per-cone kernels,
//     outputs by the per-instance kernel), so nothing must start at zero.
//   * The array, and the host staging array, are shared by every call on a
//     device: overlapping calls (two host threads, or two streams) race.
#include <cstring>
#include <mutex>

#include "../../include/clgpu.h"
#include "cones.cuh"

using namespace clgpu;

namespace {

constexpr int kMaxCones = CLGPU_MARGINS_STATIC_MAX_CONES;
// double words: cone_tmp[kMaxCones] | cone_tmp2[kMaxCones] | out[2] | pad
constexpr int kDblWords = 2 * kMaxCones + 32;
// int words, packed per call: soc_off, soc_dim, soc_inst, psd_off, psd_n,
// psd_inst (n_soc or n_psd each), then 10 range words
constexpr int kIntWords = 3 * kMaxCones + 16;
constexpr size_t kScratchWords = kDblWords + (kIntWords + 1) / 2;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_margins_scratch[kScratchWords];

int g_host_ints[kIntWords];  // host staging for the packed layout
double *g_dev_base[kMaxDevices] = {nullptr};
std::mutex g_base_mu;

int scratch_base(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return -1000 - (int)e;
  if (dev < 0 || dev >= kMaxDevices) return -1;
  std::lock_guard<std::mutex> lk(g_base_mu);
  if (!g_dev_base[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_margins_scratch);
    if (e != cudaSuccess) return -1000 - (int)e;
    g_dev_base[dev] = static_cast<double *>(p);
  }
  *out = g_dev_base[dev];
  return 0;
}

}  // namespace

extern "C" int clgpu_margins_static(int ncones, const int *types, const int *dims,
                                    const double *z, int pd, double *alpha, double *beta,
                                    clgpu_stream_t stream) {
  if (ncones < 0 || (ncones > 0 && (!types || !dims)) || !z) return -1;
  int n_soc = 0, n_psd = 0, psd_max = 1, soc_max = 0;
  for (int c = 0; c < ncones; ++c) {
    const int t = types[c], d = dims[c];
    if (t < 0 || t > 5 || d < 0) return -1;
    if (c > 0 && t < types[c - 1]) return -2;  // compositecone_type_gpu.jl:75-79
    if (t == 2) {
      ++n_soc;
      soc_max = d > soc_max ? d : soc_max;
    }
    if (t == 5) {
      if (d > kPsdMaxSide) return -3;
      ++n_psd;
      psd_max = d > psd_max ? d : psd_max;
    }
  }
  if (n_soc + n_psd > kMaxCones) return CLGPU_ERR_STATIC_TOO_LARGE;

  double *base = nullptr;
  int rc = scratch_base(&base);
  if (rc) return rc;

  // packed layout on the host staging array
  int *soc_off = g_host_ints, *soc_dim = soc_off + n_soc, *soc_inst = soc_dim + n_soc;
  int *psd_off = soc_inst + n_soc, *psd_n = psd_off + n_psd, *psd_inst = psd_n + n_psd;
  int *rng = psd_inst + n_psd;
  int row = 0, nn_begin = -1, n_nn = 0, is = 0, ip = 0;
  for (int c = 0; c < ncones; ++c) {
    const int t = types[c], d = dims[c];
    const int nv = (t == 3 || t == 4) ? 3 : (t == 5 ? d * (d + 1) / 2 : d);
    if (t == 1) {
      if (nn_begin < 0) nn_begin = row;
      n_nn += nv;
    } else if (t == 2) {
      soc_off[is] = row;
      soc_dim[is] = d;
      soc_inst[is++] = 0;
    } else if (t == 5) {
      psd_off[ip] = row;
      psd_n[ip] = d;
      psd_inst[ip++] = 0;
    }
    row += nv;
  }
  const int r10[10] = {0, n_nn, 0, n_soc, 0, 0, 0, 0, 0, n_psd};
  std::memcpy(rng, r10, sizeof(r10));
  const int n_ints = 3 * (n_soc + n_psd) + 10;

  double *dbl = base;
  int *ints = reinterpret_cast<int *>(base + kDblWords);
  ConeSet cs{};
  cs.B = 1;
  cs.soc_skip_lo = 1;  // empty skip range: the lane-group kernels take every cone
  cs.soc_skip_hi = 0;
  cs.m_total = row;
  cs.nn_begin = nn_begin < 0 ? 0 : nn_begin;
  cs.n_nn = n_nn;
  cs.n_soc = n_soc;
  cs.n_exp = 0;  // exponential and power cones contribute no margin
  cs.n_pow = 0;
  cs.n_psd = n_psd;
  int G = 2;
  while (G < soc_max && G < 32) G <<= 1;
  cs.soc_group = G;
  cs.psd_nmax = psd_max;
  cs.soc_off = ints;
  cs.soc_dim = ints + n_soc;
  cs.soc_inst = ints + 2 * n_soc;
  cs.psd_off = ints + 3 * n_soc;
  cs.psd_n = cs.psd_off + n_psd;
  cs.psd_inst = cs.psd_n + n_psd;
  const int *drng = cs.psd_inst + n_psd;
  cs.rng_nn = drng;
  cs.rng_soc = drng + 2;
  cs.rng_exp = drng + 4;
  cs.rng_pow = drng + 6;
  cs.rng_psd = drng + 8;
  cs.cone_tmp = dbl;
  cs.cone_tmp2 = dbl + kMaxCones;
  cs.inst_active = nullptr;
  double *out = dbl + 2 * kMaxCones;

  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(ints, g_host_ints, (size_t)n_ints * sizeof(int),
                                  cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return -1000 - (int)e;
  cones_margins(cs, z, pd, out, out + 1, st);
  double res[2] = {0, 0};
  e = cudaMemcpyAsync(res, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return -1000 - (int)e;
  e = cudaGetLastError();
  if (e != cudaSuccess) return -1000 - (int)e;
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return -1000 - (int)e;
  if (alpha) *alpha = res[0];
  if (beta) *beta = res[1];
  return 0;
}
