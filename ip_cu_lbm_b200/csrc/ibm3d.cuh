// Moving immersed boundary coupled to the 3-D solver (ibm3d.cu): a rigid
// sphere whose markers sit on a Fibonacci lattice, multi-direct forcing
// with the reference's 4-point Peskin kernel per axis (ref:
// function/ibm.cu:61-66 weightFunction), evaluated in index space on
// stretched axes, and an FP64 rigid-body update built on the reference's
// update_IBbody / update_IBpoint (ref: function/ibm.cu:367-447) in three
// dimensions.
#pragma once
#include <stdint.h>

namespace ipcu {
namespace ib3d {

constexpr int kThreads = 1024;
constexpr int kMaxMarkers = 1024;  // the marker arrays live in shared memory (100 B each)
constexpr int kMaxWin = 65536;  // cells of the window box (old and new footprints)

// Device-resident FP64 body state.
struct Body {
  double X[3], U[3], om[3];  // centre, velocity, angular velocity
  double R[9];               // orientation (body frame -> lab), row major
  double P[3], L[3];         // fluid momentum and angular momentum inside the body, previous step
  double Fib[3], Tib[3];     // force and torque the markers put on the fluid, previous step
  int win[6];                // window box of the last update (i0, j0, k0, wi, wj, wk); wi = 0: none
  int have_prev;
  int pad;
};

// One coupled sphere after a fluid step: the buffers of the state that step
// wrote and the body's own arrays.
struct Job {
  const float *f, *g;  // populations of the state [19][N], [7][N]
  float *F;            // its force planes [3][N] (corrected in place: the next step's velocity)
  float *fext;         // [3][N] force density on the fluid (zero outside the window)
  int nx, ny, nz;
  float c, hdt, rho0, rsal;
  const double *xc, *yc;  // cell centres along x, y (physical units)
  const float *wx, *wy;   // cell widths along x, y
  double dz, dt;
  Body *body;
  const double *r0;  // [nl][3] marker positions in the body frame
  const double *dA;  // [nl] area per marker
  int nl, iters;
  double m, I, rho_s, rho_f, grav, radius;
  // global scratch of the window (the marker arrays and the pair offsets
  // are in the kernel's shared memory)
  int *cur;                // [kMaxWin + 1] fill cursors of the pair lists
  int *list;               // [64 nl] pairs (64 marker + node) by window cell
  float *wu, *wf, *wj;     // [3][kMaxWin] velocity u*, accumulated force density, momentum c j per window cell
  float *wh, *wv;          // [kMaxWin] dt / 2 rho and cell volume
  unsigned *status;
};

int launch(const Job &j, cudaStream_t s);
int prepare();

}  // namespace ib3d
}  // namespace ipcu
