// sn_exec.cuh -- device state and entry points of the supernodal LDL^T
// (supernodal.cu); the plan it runs is built by supernodal.cpp.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "devbuf.hpp"
#include "supernodal.hpp"

namespace clgpu {

struct KKTDev;
struct LDLParams;

// Plan arrays on the device (see SnPlan) plus the numeric storage.
struct SnDev {
  const int *inst, *col0g, *ncol, *nrow, *u0, *ld, *cbase, *fix_off, *rel_off, *ch_ptr, *ch,
      *uoff, *fidx, *rel, *acol;
  const long long *foff, *woff, *soff;
  const int2 *amap;
  const int4 *tasks;
  const int *cl_ptr;   // per chunk of a blocked front: its children in clist
  const int4 *clist;   // {child, q_begin, q_end}
  void *F;       // fronts (T)
  void *W;       // factor workspace of blocked fronts (T): dinv, W
  double *S;     // solve workspace of blocked fronts: work vector, partial sums
  double *U;     // forward-substitution contributions, nrow per supernode
  double *Dinv;  // [global vector index] 1 / pivot
  double *eps;   // [B] static regularisation of the last factorisation
  int *srun;     // [B] instances taking part in the current solve sweep
  unsigned long long *nrm;  // [2 B] |b|_inf and |e|_inf (bit patterns of non-negative doubles)
  // refinement vectors, indexed by global vector index - vbase
  double *b, *x, *xn, *e, *y;
  const int *vinst;  // [vcount] instance of the vector entry, -1 when not in the plan
  int vbase, vcount;
};

struct SnExec {
  SnDev d{};
  std::vector<SnLaunch> fact, fwd, bwd;
  std::vector<int> insts;  // instances of the plan
  int *d_insts = nullptr;
  int B = 0;
  int small_smem = 0;  // elements of the largest small front
  bool fp32 = false;
  double flops = 0;    // factorisation flops (padded GEMM tiles in full)
  int *h_srun = nullptr;                // pinned [B]
  int *h_flags = nullptr;               // pinned [B]
  unsigned long long *h_nrm = nullptr;  // pinned [2 B]
  int *d_flags = nullptr;               // [B]
  long long launches = 0;               // kernel launches issued (statistics)
  // one substitution pass (forward, D^-1, backward) as a CUDA graph,
  // captured on first use on a private stream and replayed on the caller's
  // stream (not used while profiling, which brackets every launch)
  cudaStream_t cap = nullptr;
  cudaGraphExec_t g_pass = nullptr;
  long long pass_launches = 0;
  bool graph_failed = false;
  // refinement statistics since profiling was switched on: solves, sweeps,
  // solves that stopped above the tolerance, and the worst such final
  // |e|_inf / (abstol + reltol |b|_inf)
  long long ir_solves = 0, ir_sweeps = 0, ir_unconverged = 0;
  double ir_worst = 0.0;
  // profiling: every launch bracketed by CUDA events, device time and
  // algorithmic flops summed per launch kind (SnLaunchKind)
  struct Prof {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    std::vector<int> kinds;  // kind of event pair k (events 2k, 2k + 1)
    double ms[SN_KINDS] = {}, flops[SN_KINDS] = {};
    long long calls[SN_KINDS] = {};
  } prof;
  ~SnExec();
};
// profiling on / off (turning it on clears the totals) and the totals
void sn_set_profiling(SnExec &ex, bool on);
void sn_get_profile(const SnExec &ex, double *ms, double *flops, long long *calls);

// Uploads the plan and allocates the fronts and workspaces (arena-owned).
// false when an allocation fails.
bool sn_exec_create(const SnPlan &plan, bool fp32, int B, int vbase, int vcount,
                    const std::vector<int> &vinst, DevArena &A, SnExec &ex);
// Numeric refactorisation of the plan's instances with run[i] != 0 (the KKT
// values in k.Kx, static and dynamic regularisation as in p); clears ok[i] on
// a non-finite pivot; eps_out[i] receives the static regulariser.
void sn_factor(SnExec &ex, const KKTDev &k, const LDLParams &p, const int *run, int *ok,
               double *eps_out, cudaStream_t st);
// Solve with iterative refinement for the plan's instances with run[i] and
// ok[i]; same contract as ldl_solve.  Synchronises the stream between
// refinement sweeps.
void sn_solve(SnExec &ex, const KKTDev &k, const LDLParams &p, const int *run, const double *rx,
              const double *rz, double *lx, double *lz, int *ok, cudaStream_t st);

}  // namespace clgpu
