// cones.cuh -- launchers for the per-cone kernels (cones.cu).
//
// One launcher per CompositeConeGPU operation of the reference
// (src/gpucones/coneops_compositecone_gpu.jl).  Each launcher covers every
// cone type of every instance of a batch.  Per-instance scalars are device
// arrays indexed by instance; nothing is read back to the host.
#pragma once
#include "common.cuh"

#include <vector>

namespace clgpu {

// Second-order cones of dim <= kSocTileMaxDim can be processed in
// shared-memory tiles by the per-iteration operations below: a tile is a run
// of consecutive cones with contiguous rows (at most C cones and 8*C rows,
// C = 32, 64 or 128 = the block size), staged with coalesced loads and
// stores, one thread per cone.  The alternative is a lane group per cone.
// Both evaluate the same formulas with sums in the same butterfly order, so
// the choice (made per cone set by cones_autotune) does not change results.
constexpr int kSocTileMaxDim = 16;
constexpr int kSocTileShapes = 3;  // v = 1..3: 32, 64, 128 cones per tile
__host__ __device__ constexpr int soc_tile_cones(int v) { return 32 << (v - 1); }
__host__ __device__ constexpr int soc_tile_rows(int v) { return 8 * soc_tile_cones(v); }
enum SocOp {
  kSocUpdateScaling = 0,
  kSocAffineDs,
  kSocCombined,
  kSocDsOffset,
  kSocStep,
  kSocMulHs,
  kSocOps
};
// Tile list [c0, c1, c0, c1, ...] over the cones of dim <= kSocTileMaxDim
// among n cones (rows off[k] .. off[k]+dim[k]), at most max_cones cones and
// max_rows rows per tile.
std::vector<int> soc_tiles(const int *off, const int *dim, int n, int max_cones, int max_rows);
// Default launch shapes of a cone set (before or without tuning).
void cones_default_shapes(ConeSet &cs);
// Times the candidate launch shapes of the nonnegative and SOC kernels on
// this cone set (scratch state and vectors, nothing of cs is written but
// its shape fields) and keeps the fastest; without room for the scratch it
// keeps the default shapes.  Returns 0 or -1000 - cudaError.
int cones_autotune(ConeSet &cs, cudaStream_t st);

// update_scaling!  (coneops_compositecone_gpu.jl:185).  mu/scaling are
// per-instance device arrays; scale_ok[i] is cleared to 0 on failure.
void cones_update_scaling(const ConeSet &cs, const double *s, const double *z,
                          const double *mu, const int *scaling, int *scale_ok,
                          cudaStream_t st);
// Hs refresh fused with the KKT scatter (get_Hs! + kktsolver_update!):
// writes -Hs into kkt_vals at the positions in map.
void cones_refresh_kkt(const ConeSet &cs, const KKTMapDev &map,
                       double *kkt_vals, cudaStream_t st);
// get_Hs! into a packed Hsblocks vector laid out like the reference
// (blk_off[c] per cone of each type, see capi).  Used by the cone-level ABI.
void cones_get_Hs(const ConeSet &cs, const int *nn_blk, const int *soc_blk,
                  const int *exp_blk, const int *pow_blk, const int *psd_blk,
                  double *Hs, cudaStream_t st);
void cones_mul_Hs(const ConeSet &cs, double *y, const double *x,
                  cudaStream_t st);
void cones_affine_ds(const ConeSet &cs, double *ds, const double *s,
                     cudaStream_t st);
void cones_combined_ds_shift(const ConeSet &cs, double *shift,
                             const double *step_z, const double *step_s,
                             const double *sigma_mu, cudaStream_t st);
void cones_ds_from_dz_offset(const ConeSet &cs, double *out, const double *ds,
                             const double *z, cudaStream_t st);
// symmetric-cone step length: atomically mins into alpha[i] (pre-set to the
// instance's alpha_max).
void cones_step_length_sym(const ConeSet &cs, const double *dz,
                           const double *ds, const double *z, const double *s,
                           double *alpha, cudaStream_t st);
// asymmetric cones: backtracking from alpha_start[i]; mins into alpha[i]
void cones_step_length_asym(const ConeSet &cs, const double *dz,
                            const double *ds, const double *z, const double *s,
                            const double *alpha_start, double *alpha,
                            double backtrack, double alpha_min,
                            cudaStream_t st);
// compute_barrier: adds each instance's cone barrier at alpha[i] into bar[i]
// (deterministic: per-cone values reduced per instance in a fixed order)
void cones_barrier(const ConeSet &cs, const double *z, const double *s,
                   const double *dz, const double *ds, const double *alpha,
                   const int *bt_active, double *bar, cudaStream_t st);
// margins: min margin into amin[i], sum of positive margins into asum[i]
// (deterministic per-instance reduction; outputs overwritten)
void cones_margins(const ConeSet &cs, const double *z, int pd, double *amin,
                   double *asum, cudaStream_t st);
void cones_scaled_unit_shift(const ConeSet &cs, double *z,
                             const double *alpha, int pd, cudaStream_t st);
void cones_unit_initialization(const ConeSet &cs, double *z, double *s,
                               cudaStream_t st);
void cones_set_identity_scaling(const ConeSet &cs, cudaStream_t st);

}  // namespace clgpu
