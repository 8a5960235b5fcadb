// supernodal.hpp -- supernodal (multifrontal) LDL^T for the large problems.
//
// The reference factors a large KKT matrix with cuDSS: analysis once
// (src/kktsolvers/gpu/directldl_cudss.jl:20-23), numeric refactorisation
// every IPM iteration (:37-46) and a solve (:50-59), in FP64 or, for
// :cudssmixed, in FP32 (directldl_mixed_cudss.jl:24-78).  cuDSS is not
// available here; this is the project's own sparse direct solver for the
// instances too large for the single-warp kernels.
//
// Host side (supernodal.cpp): approximate minimum degree ordering
// (amd.cpp), elimination tree and postorder, column counts, fundamental
// supernodes merged by a relaxed-amalgamation rule, the row structure of
// every supernode, and the device plan: front layout, assembly maps, child
// -> parent relative indices and the per-level launch schedule.
//
// Device side (supernodal.cu): level by level from the leaves, every front
// (the supernode's pivot columns plus its row structure, dense, column-major)
// is assembled from the KKT values and the children's Schur complements
// (extend-add), and its pivots are eliminated.  Fronts of at most
// kSnSmallMax rows are assembled and factored by one block in shared memory;
// larger fronts are padded to kSnNB-column panels and factored panel by
// panel: the diagonal block by one block, the rows below it by triangular
// substitution, and the trailing matrix by a rank-kSnNB update (FP64
// tensor-core MMA, or FP32 FMA in the mixed-precision form).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace clgpu {

constexpr int kSnNB = 128;       // panel width and tile edge of the blocked fronts
constexpr int kSnSmallMax = 128;  // fronts with at most this many rows: one block, shared memory

// Supernodal symbolic factorisation of one matrix (indices are positions in
// the permuted matrix).
struct SnSymbolic {
  int N = 0;
  std::vector<int> col0;    // [ns + 1]: supernode s owns pivot columns [col0[s], col0[s + 1])
  std::vector<int> parent;  // [ns]: parent supernode, -1 for a root
  std::vector<int> rptr;    // [ns + 1]
  std::vector<int> rows;    // row structure of s below its last column, sorted
  double nnz_l = 0;         // entries of L including the amalgamation's explicit zeros
  double flops = 0;         // sum over columns of (entries below the diagonal)^2
  int ns() const { return (int)parent.size(); }
};

// Fill-reducing ordering and supernodal symbolic factorisation of a
// symmetric pattern given as a CSR graph (self loops and repeats allowed).
// perm[k] = original index eliminated k-th.  Returns false (with *err) on
// a size overflow.
bool sn_analyse(int N, const std::vector<int> &xadj, const std::vector<int> &adj,
                std::vector<int> &perm, SnSymbolic &sym, std::string *err);

// ------------------------------------------------------------ device plan
// Pivot columns of a blocked front are padded to a multiple of kSnKPad with
// dummy pivots (unit diagonal, no coupling) and its row structure to a
// multiple of kSnNB, so every trailing region is a whole number of
// kSnNB x kSnNB tiles: the first panel takes u0 mod kSnNB columns (when
// nonzero), every later panel kSnNB.
constexpr int kSnKPad = 16;
constexpr int kSnAsmCols = 32;  // parent columns per assembly task

struct SnPair {
  int x, y;
};
struct SnQuad {
  int x, y, z, w;
};

// Launches of the factorisation and solve schedules; tasks[begin, begin +
// count) are the launch's blocks (or warps, for the small-front solves).
enum SnLaunchKind : int {
  SN_SMALL_FACTOR = 0,  // {s}: assemble + factor a small front in shared memory
  SN_ASSEMBLE,          // {s, c_begin, c_end, chunk}: zero + assemble columns of a blocked front
  SN_DIAG,              // {s, k | K << 16}: factor the K x K diagonal block
  SN_TRSM,              // {s, k | K << 16, r0}: rows r0..r0+127 of the panel: W = A L11^-T
                        //   by substitution, L = W D^-1
  SN_UPDATE,            // {s, k | K << 16, r0, c0}: 128 x 64 tile (r0, c0) -= L(r0 rows) W(c0 rows)^T
  SN_FWD_SMALL,         // {s}: forward substitution of a small front (one warp)
  SN_FWD_GATHER,        // {s, c_begin, c_end, chunk}: positions of a blocked front's work vector
  SN_FWD_DIAG,          // {s, k | K << 16}: v(panel) <- L11^-1 v(panel)
  SN_FWD_GEMV,          // {s, k | K << 16, r0}: v(r0 rows) -= L(r0 rows, panel) v(panel)
  SN_FWD_SCATTER,       // {s}
  SN_BWD_SMALL,         // {s}
  SN_BWD_GATHER,        // {s}
  SN_BWD_PARTIAL,       // {s, k | K << 16, r0}: L(r0 rows, panel)^T v(r0 rows)
  SN_BWD_DIAG,          // {s, k | K << 16}: v(panel) <- L11^-T (v(panel) - partial sums)
  SN_BWD_SCATTER,       // {s}
  SN_KINDS
};
struct SnLaunch {
  int kind, begin, count, smem;
  double flops;  // algorithmic floating-point operations of the launch (factorisation)
};

// One instance handed to the plan builder.
struct SnInstance {
  const SnSymbolic *sym;
  const int *Kp, *Kj;  // permuted full KKT of the instance, CSR, local indices
  long long kbase;     // global position of the instance's first KKT value
  int vbase;           // global index of the instance's first vector entry
  int inst;            // instance number in the batch
};

// Everything the device needs, concatenated over the instances.  Front
// layout of supernode s (column-major, leading dimension ld[s]):
//   [0, ncol)          pivot columns (global vector index col0g + c)
//   [ncol, u0)         dummy pivots (blocked fronts only)
//   [u0, u0 + nrow)    the row structure: the update (Schur complement) region
//   [u0 + nrow, ld)    zero padding (blocked fronts only)
// Small fronts (ncol + nrow <= kSnSmallMax) have u0 = ncol and ld = ncol + nrow.
struct SnPlan {
  int ns = 0;
  std::vector<int> inst, col0g, ncol, nrow, u0, ld, large, cbase, fix_off, rel_off, ch_ptr,
      uoff;
  std::vector<long long> foff;  // front offsets (elements, multiples of 32)
  std::vector<long long> woff;  // factor workspace of blocked fronts: dinv (kSnNB), W (ld x kSnNB)
  std::vector<long long> soff;  // solve workspace of blocked fronts: v (ld), partial sums (ld)
  std::vector<int> ch;          // children, in order
  std::vector<int> fidx;        // front position -> global vector index (-1 none)
  std::vector<int> rel;         // struct row k of s -> position in the parent's front
  std::vector<int> acol;        // [sum ncol + 1] start of pivot column (cbase[s] + c) in amap
  std::vector<SnPair> amap;     // {global KKT position, front offset} of original entries
  // children touching each kSnAsmCols-wide chunk of a blocked front's
  // positions, in child order: {child, q_begin, q_end} (the child's row
  // structure entries q whose parent positions fall in the chunk); chunk k
  // of front s is chunk_off[s] + k, its entries clist[cl_ptr[..]..)
  std::vector<int> chunk_off, cl_ptr;
  std::vector<SnQuad> clist;
  std::vector<SnQuad> tasks;
  std::vector<SnLaunch> fact, fwd, bwd;
  std::vector<int> insts;       // the instances of the plan
  long long f_elems = 0, w_elems = 0, s_elems = 0, u_elems = 0;
  int small_smem_max = 0;       // largest small front, elements
  double flops = 0;             // factorisation flops of the padded fronts (sum over launches)
};

// Builds the plan; false (with *err) on an index overflow.
bool sn_build_plan(const std::vector<SnInstance> &in, SnPlan &plan, std::string *err);

// Host replay of the device factorisation and solve on the plan (FP64):
// factors the KKT values Kx (global positions, the diagonal shifted by
// eps * Dsign) and solves K x = b for the plan's instances; returns the
// relative residual ||K x - b||_inf / ||b||_inf of a test right-hand side.
// Needs no GPU; used to check every map before a kernel reads it.
double sn_host_check(const SnPlan &plan, const std::vector<int> &Kp, const std::vector<int> &Kj,
                     const std::vector<double> &Kx, const std::vector<signed char> &Dsign,
                     const std::vector<int> &voff, double eps);

}  // namespace clgpu
