// setup.hpp -- host-side, once-per-problem preparation for libclgpu.
//
// For every instance: data equilibration (Ruiz), cone placement into the
// type-major batch layout, full KKT pattern with the sparse second-order-cone
// expansion, fill-reducing ordering, symbolic LDL^T and the index maps used
// by the device refresh/solve kernels.  Instances are prepared in parallel on
// host threads and then concatenated into flat arrays that are uploaded once.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/clgpu.h"
#include "supernodal.hpp"

namespace clgpu {

struct HostCSC {
  int m = 0, n = 0;
  std::vector<int> p, i;
  std::vector<double> x;
};

// One prepared instance (local indices).
struct Prepared {
  int n = 0, m = 0, N = 0;  // N = n + m + 2 * n_sparse_soc
  std::string error;
  // equilibrated data
  std::vector<double> q, b;        // b in user row order
  std::vector<double> d, e;        // equilibration (e in user row order)
  double c = 1.0, normq = 0, normb = 0;
  HostCSC Pfull;                   // full symmetric, equilibrated (CSC)
  HostCSC A;                       // equilibrated A (CSC, user row order)
  int p_nnz = 0;                   // nnz of the user's upper-triangular P
  // cones in type-major local order
  std::vector<int> ctype, cdim;
  std::vector<double> cparam;
  std::vector<int> cstart;         // local type-major row of the cone's first element
  std::vector<int> user_row_of;    // local type-major row -> user row
  std::vector<int> type_rows;      // [6] row counts per type
  std::vector<int> type_cones;     // [6] cone counts per type
  bool symmetric = true;
  int degree = 0;
  // KKT (permuted full CSR, local positions)
  std::vector<int> perm, iperm;
  std::vector<int> Kp, Kj, Kdiag;
  std::vector<double> Kx;          // constant P/A entries (others 0)
  std::vector<signed char> Dsign;  // permuted
  std::vector<int> Lp, Li, Rp, Rk, Rpos;
  std::vector<int> lvl_ptr, lvl_nodes;  // elimination-tree levels (leaves first)
  // Large instances (work vector beyond the single-warp kernels' budget)
  // take the supernodal factorisation: AMD ordering, supernodal symbolic
  // structure in sym, and no scalar structures (Lp, Rp zero, Li, Rk, Rpos
  // and the levels empty).
  bool supernodal = false;
  SnSymbolic sym;
  // refresh positions (local CSR positions)
  std::vector<int> nn_pos;                   // per NN row (type-major order)
  std::vector<int> socd_pos;                 // dense SOC triu pairs (concat over cones)
  std::vector<int> socd_start;               // per SOC cone start (entries) or -1
  std::vector<int> socs_diag, socs_uv;       // per SOC row (type-major), -1 if dense
  std::vector<int> socs_D;                   // per SOC cone 2 (or -1)
  std::vector<int> exp_pos, pow_pos;         // 12 per cone
  std::vector<int> psd_pos, psd_start;       // pairs per triu entry, start per cone
  // value updates (update_data!): for every entry of the caller's P (CSC
  // order, entries below the diagonal included and ignored), the positions
  // of the value in the full symmetric P (two for off-diagonals, else -1) and
  // in the KKT matrix (two / one, -1 when ignored); for every entry of A its
  // two KKT positions.  updatable is false when the caller's matrices held
  // repeated entries (their values were summed at setup).
  std::vector<int> pmap;   // 4 per caller P entry: pfull1, pfull2, kkt1, kkt2
  std::vector<int> pxy;    // 2 per caller P entry: local (row, col), -1 if ignored
  std::vector<int> amapk;  // 2 per A entry: kkt1, kkt2
  int p_user_nnz = 0;
  bool updatable = true;
  // equilibration left to the device (SetupOptions::defer_equilibration):
  // d, e = 1, c = 1 and the data unscaled here
  bool eq_deferred = false;
  // for gathering rhs / scattering solution: permuted k -> local original idx
  // (0..n-1 x, n..n+m-1 z type-major local row, >= n+m extra)
};

struct SetupOptions {
  int soc_threshold = 5;
  int equilibrate_enable = 1, equilibrate_max_iter = 10;
  double equilibrate_min_scaling = 1e-4, equilibrate_max_scaling = 1e4;
  // leave the Ruiz equilibration (and so the KKT values) to the device when
  // the caller's P and A columns are sorted without repeated entries
  bool defer_equilibration = false;
};

bool prepare_instance(const clgpu_problem &pb, const SetupOptions &opt,
                      Prepared &out);

// fill-reducing ordering of a symmetric pattern given as an adjacency list
// (no self loops); returns perm (perm[k] = original index eliminated k-th)
std::vector<int> amd_order(int n, std::vector<std::vector<int>> &adj);
// nested-dissection ordering (minimum degree on the small parts); same
// contract as amd_order
std::vector<int> nd_order(int n, std::vector<std::vector<int>> &adj);
// the same on a CSR graph (repeated neighbours allowed; rows are sorted and
// deduplicated in place)
std::vector<int> nd_order_csr(int n, std::vector<int> &xadj, std::vector<int> &adjncy);
// approximate minimum degree on the quotient graph (amd.cpp): the
// fill-reducing ordering of the supernodal factorisation; CSR graph,
// repeated neighbours and self loops allowed; same contract as amd_order
std::vector<int> amd_order_qg(int n, const std::vector<int> &xadj, const std::vector<int> &adj);

}  // namespace clgpu
