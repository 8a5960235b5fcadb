// ldl.cuh -- batched sparse LDL^T of the quasi-definite KKT systems.
//
// Stands in for the reference's cuDSS calls (src/kktsolvers/gpu/
// directldl_cudss.jl:30-59 and directldl_mixed_cudss.jl:42-78), which are not
// available in this environment.  The host computes a fill-reducing ordering
// and the symbolic factorisation once per instance (setup.cpp); the device
// refactors every IPM iteration and solves with iterative refinement
// (kktsolver_directldl_gpu.jl:300-409).
#pragma once
#include "common.cuh"

namespace clgpu {

struct SnExec;

struct KKTDev {
  int B;
  const int *N;     // [B] KKT dimension of each instance
  const int *voff;  // [B+1] offsets of per-instance vectors (sum of N)
  const int *poff;  // [B]   offsets into the (N+1)-long pointer arrays
  // permuted full KKT (both triangles), CSR with global positions
  const int *Kp, *Kj;
  double *Kx;
  const int *Kdiag;          // [sum N] position of the diagonal of each row
  const signed char *Dsign;  // [sum N] +1 / -1
  const int *gsrc;           // [sum N] rhs gather / solution scatter codes
  // factor L (strict lower, CSC with global positions) and D
  const int *Lp, *Li;
  void *Lx, *D, *Dinv;  // double or float (mixed precision)
  // row pattern of L: for column j the list (k, pos of L(j,k))
  const int *Rp, *Rk, *Rpos;
  // elimination-tree levels: nodes of level l of instance i are
  // lvl_nodes[voff[i] + lvl_ptr[lvl_off[i] + l] .. lvl_ptr[lvl_off[i] + l + 1])
  const int *lvl_off, *nlev, *lvl_ptr, *lvl_nodes;
  // substitution schedules, one int4 per node:
  //   fsched[voff[i] + t] = {node, Rp[node], Rp[node+1], 0} in level order
  //     (leaves first);
  //   bsched[voff[i] + t] = {node, Lp[node], Lp[node+1], 0} in backward order
  //     (root level first: level l occupies [N - lvl_ptr[l+1], N - lvl_ptr[l]))
  const int4 *fsched, *bsched;
  // copy of L's values in row-pattern order (LxR[r] = Lx[Rpos[r]]), written at
  // the end of every factorisation so the forward substitution reads L rows
  // contiguously; same element type as Lx
  void *LxR;
  // Single-warp instances substitute by streaming nonzeros in level order.
  // Forward stream: the row patterns of the nodes of level 0, 1, ... (node
  // by node), entry {seg = row node i, idx = column k}; backward stream: the
  // columns of the nodes from the root level down, entry {seg = column node
  // j, idx = row i}.  Both occupy the instance's L positions [Lp[0], Lp[N]);
  // flev / blev (nlev + 1 per instance, at lvl_off) give each level's start
  // in processing order.  LxF / LxB hold L's values in stream order (copied
  // from Lx[fpos] / Lx[bpos] after every factorisation).  kent is {row,
  // column} of every KKT entry (CSR order) for the refinement residual.
  const int2 *fent, *bent, *kent;
  const int *fpos, *bpos, *flev, *blev;
  void *LxF, *LxB;
  // Entry encoding of the three streams (single-warp instances only):
  //   .x = segment | min(position in segment, kSPosMax) << 16 | last << kSLastBit
  //   .y = gathered index
  // Chunk tables: a pass is a list of chunks of <= kSChunk consecutive
  // entries of one level, encoded as described below.  Instance i's chunks of
  // the forward, backward and residual passes are fch[fch_off[i] ..
  // fch_off[i+1]) etc.
  const int *fch, *bch, *kch, *fch_off, *bch_off, *kch_off;
  // Streamed factorisation (single-warp instances whose N + nnz(L) FP64
  // values fit in shared memory, fstream[i] = 1), one block of kFactorWarps
  // warps per instance.  The block keeps U = L D (column j of L times d_j)
  // and, once pivot j is final, 1/d_j in shared memory.  Per level of the
  // elimination tree the op stream lists, sorted by target, every update
  //     V[t] -= V[a] * V[b] * V[k]   (U(i,k) U(j,k) / d_k into U(i,j) or d_j)
  // as one 8-byte op word (fop_pack: t, a, b, k, position in segment, last),
  // split into kFactorWarps parts at target boundaries (part w for warp w),
  // followed by the level's pivots (t = j, a = sign + 1), also in
  // kFactorWarps parts.
  // Indices address the shared array [d or 1/d (N) | U (nnz(L))].  Warp w of
  // instance i reads its chunk words foch[fwoff[(kFactorWarps+1) i + w] ..
  // fwoff[(kFactorWarps+1) i + w + 1]) (start relative to fop_base[i], pivot
  // chunks flagged); flcnt[(lvl_off[i] + l) kFactorWarps + w] = its number of
  // op chunks | pivot chunks << 16 at level l.  The block synchronises after
  // each level's updates and after its pivots.  Lkpos: KKT position of every
  // L entry (-1: structural zero).  fs_inst lists the fs_count streamed
  // instances by decreasing shared-memory need (block b factors fs_inst[b]);
  // fs_smem bytes per block.
  const int *fstream, *fop_base, *foch, *fwoff, *flcnt, *Lkpos, *fs_inst;
  const uint2 *fop;
  int has_fstream, fs_count, fs_smem;
  // Packing of single-warp solves into blocks of kSolveWarps warps (first fit
  // by decreasing shared-memory need: the work vector y, N FP64 values, plus
  // the warp's ring): warp w of block b solves spack_inst[kSolveWarps b + w]
  // (-1: idle) with its shared memory at byte spack_off[...]; spack_smem
  // bytes per block.
  const int *spack_inst, *spack_off;
  int spack_blocks, spack_smem;
  // the same for solves of two right-hand sides at once (two work vectors)
  const int *spack2_inst, *spack2_off;
  int spack2_blocks, spack2_smem;
  // profiling only (else null): per instance, algorithmic bytes moved by the
  // factorisations [0, B), the one-side solves [B, 2B) and the two-side
  // solves [2B, 3B) of the profiled solve
  double *prof_bytes;
  // [B] kernel class: 1 = single warp (work vector in shared memory, the
  // streams above), 2 = block kernels with global scratch, 3 = supernodal
  // (sn below; no scalar factor structures)
  const int *cls;
  // supernodal factorisation of the class-3 instances (host object; null
  // when there are none)
  SnExec *sn;
  int max_small_N;       // largest N among single-warp (shared memory) instances
  int has_small, has_large;
  int has_small_legacy;  // single-warp instances without a streamed factorisation
  // scratch (global, per instance, sum N each)
  double *w;       // dense factor accumulator (large instances)
  double *yf;      // substitution work vector (large instances)
  // FP32-stored factor only (null otherwise): the FP64 factor values and
  // pivots the factorisation itself runs on; the solves read the FP32 copy
  double *Lacc;
  double *Dacc;
  // single-warp solve scratch per instance (sum N each): right-hand side b,
  // accepted iterate x and residual e of the first and the second side
  double *b, *x, *e, *b2, *x2, *e2;
  double *dx;
};

// Stream chunking shared by the setup and the kernels.  A chunk is a run of
// consecutive entries of one level; lane l of the warp holds K consecutive
// entries K l .. K l + K - 1 of it.  Chunk words carry the chunk's start
// relative to the instance's stream base (bits 0..21), its "scan steps"
// (bits 22..24) and its count - 1 (from bit 25).  Scan steps (0..5) is how
// many doubling steps of the segmented warp scan the chunk needs: the steps
// d = 1, 2, 4, ... up to the farthest any lane reaches back to the lane that
// holds the start of its last entry's segment; later steps would add
// nothing.  Streams of a single-warp instance are therefore at most
// kStartMask entries long (longer ones take the block kernels).
constexpr int kFRingSlots = 2;         // factorisation chunks in flight per warp (power of two)
constexpr int kSRingSlots = 2;         // solve chunks in flight per warp (power of two)
constexpr int kSolveWarps = 4;         // instances per single-warp-solve block
constexpr int kSolveBlocksPerSM = 4;   // solve blocks resident per SM (register budget)
constexpr int kSolveSmemMax = 200 * 1024;  // dynamic shared memory cap of a solve block
constexpr int kStepShift = 22;
constexpr int kCntShift = 25;
constexpr unsigned kStartMask = (1u << 22) - 1u;
// Substitution and residual streams (single-warp solve): K = kSK entries per
// lane; entry word segment (bits 0..15) | min(position in segment, kSPosMax)
// << 16 | last-of-segment << kSLastBit; count - 1 in 7 bits.
constexpr int kSK = 4;
constexpr int kSKShift = 2;
constexpr int kSChunk = 32 * kSK;
constexpr int kSPosMax = 127;
constexpr int kSLastBit = 23;
static_assert((1 << kSKShift) == kSK && kSPosMax + 1 >= kSChunk, "solve chunk layout");
// Factorisation op streams: K = 2 entries per lane; chunk words carry the
// count - 1 in 6 bits; bit 31 marks a pivot chunk.
constexpr int kChunk = 64;
constexpr int kFactorWarps = 4;        // warps per streamed-factorisation block (one instance)
constexpr int kPosMax = 63;
// One op in 8 bytes: four 14-bit positions in the instance's shared work
// vector (the streamed path holds at most 96 KB of it, 12288 FP64 values, so
// every position is below 2^14), min(position in segment, kPosMax) in 6 bits
// and the last-of-segment bit.  x: t | a << 14 | b << 28 (low 4 bits of b);
// y: b >> 4 | k << 10 | pos << 24 | last << 30.
constexpr int kFopBits = 14;
constexpr int kFopMaxPos = 1 << kFopBits;
__host__ __device__ __forceinline__ uint2 fop_pack(int t, int a, int b, int k, int pos,
                                                   int last) {
  uint2 w;
  w.x = (unsigned)t | ((unsigned)a << 14) | ((unsigned)b << 28);
  w.y = ((unsigned)b >> 4) | ((unsigned)k << 10) | ((unsigned)pos << 24) | ((unsigned)last << 30);
  return w;
}
__host__ __device__ __forceinline__ int fop_t(uint2 w) { return (int)(w.x & 0x3fffu); }
__host__ __device__ __forceinline__ int fop_a(uint2 w) { return (int)((w.x >> 14) & 0x3fffu); }
__host__ __device__ __forceinline__ int fop_b(uint2 w) {
  return (int)(((w.x >> 28) | (w.y << 4)) & 0x3fffu);
}
__host__ __device__ __forceinline__ int fop_k(uint2 w) { return (int)((w.y >> 10) & 0x3fffu); }
__host__ __device__ __forceinline__ int fop_pos(uint2 w) { return (int)((w.y >> 24) & 63u); }
__host__ __device__ __forceinline__ int fop_last(uint2 w) { return (int)((w.y >> 30) & 1u); }

// Scan steps of a chunk of cnt entries, K per lane, whose segment positions
// are pos(e) (clamped at or above the chunk length): lane l reaches back
// min(l, l - floor((K l + K - 1 - p) / K)) lanes, p = pos(K l + K - 1) > 0.
template <int K, typename PosOf>
inline int chunk_scan_steps(int cnt, PosOf pos) {
  int reach = 0;
  for (int l = 0; K * l + K - 1 < cnt; ++l) {
    const int p = pos(K * l + K - 1);
    if (p > 0) {
      const int a = K * l + K - 1 - p;
      int r = l - (a >= 0 ? a / K : -((-a + K - 1) / K));
      if (r > l) r = l;
      if (r > reach) reach = r;
    }
  }
  int steps = 0;
  for (int d = 1; d <= 16 && d <= reach; d <<= 1) ++steps;
  return steps;
}

struct LDLParams {
  int static_reg;
  double static_c, static_prop;
  int dyn_reg;
  double dyn_eps, dyn_delta;
  int ir_enable, ir_maxiter;
  double ir_reltol, ir_abstol, ir_stopratio;
};

// numeric refactorisation of every instance with run[i] != 0; sets
// ok[i] = 0 if a pivot is not finite; eps_out[i] receives the static
// regulariser used (diagonal_regularizer of the reference).  fp32 stores the
// factor in FP32; arith32 (with fp32) also eliminates in FP32 arithmetic,
// otherwise the elimination is FP64.
void ldl_factor(const KKTDev &k, bool fp32, const LDLParams &p, const int *run,
                int *ok, double *eps_out, cudaStream_t st, bool arith32 = false);
// solve K [lx; lz; *] = [rx; rz; 0] with iterative refinement for every
// instance with run[i] != 0.  rx/lx are indexed by global x index, rz/lz by
// global s/z row; lx or lz may be null.  ok[i] cleared on non-finite results.
void ldl_solve(const KKTDev &k, bool fp32, const LDLParams &p, const int *run,
               const double *rx, const double *rz, double *lx, double *lz,
               int *ok, cudaStream_t st);
// two right-hand sides with the same factor in one launch: side 0 (rx0, rz0)
// -> (lx0, lz0), side 1 likewise; each result is exactly that of ldl_solve
void ldl_solve2(const KKTDev &k, bool fp32, const LDLParams &p, const int *run,
                const double *rx0, const double *rz0, double *lx0, double *lz0,
                const double *rx1, const double *rz1, double *lx1, double *lz1, int *ok,
                cudaStream_t st);

}  // namespace clgpu
