// equilibrate.cuh -- device equilibration and KKT value assembly
// (equilibrate.cu).
#pragma once
#include <cuda_runtime.h>

namespace clgpu {

// Device arrays of a batch (global indices as in ipm.cu's Dev): P full
// symmetric stored by columns, A by rows, A' by rows (= A's columns).
struct EqDev {
  int B, nx, mz;
  const int *xoff;               // [B + 1]
  const int *col_inst, *row_inst;
  const int *Pp, *Pj;
  double *Px;
  const int *Ap, *Aj;
  double *Ax;
  const int *Atp, *Atj;
  double *Atx;
  double *q, *b, *negq;
  double *d, *dinv, *e, *einv, *c;  // scalings (start at 1) and their inverses
  double *dw, *ew;                  // work [nx], [mz]
  double *ct;                       // work [B]
  int *cflag;                       // work [B]
  const int *on;                    // [B] instances equilibrated here
  const int2 *rcone;                // (first global row, rows) of every rectified cone
  int nrc;
};

struct EqParams {
  int enable, max_iter;
  double smin, smax;
};

// Ruiz equilibration, cost scaling, rectification, inverses and -q for the
// instances with on[i], then their P and A values written into Kx through
// update_data!'s maps (pmap / amap: full-P or A' position and the two KKT
// positions of every caller entry; pxy / axy: global row and column).
void equilibrate_on_device(const EqDev &q, const EqParams &p, const int4 *pmap,
                           const int2 *pxy, long long np, const int4 *amap, const int2 *axy,
                           long long na, double *Kx, cudaStream_t st);

}  // namespace clgpu
