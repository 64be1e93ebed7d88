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

constexpr int kThreads = 1024;    // the set-up and the final body step (one CTA each)
constexpr int kMaxMarkers = 1024;
constexpr int kMaxWin = 65536;    // cells of the window box (old and new footprints)
constexpr int kSlots = 64;        // (marker, node) contributions a window cell may hold
constexpr int kMaxBins = 32768;   // stencil-origin bins
constexpr int kParts = 256;       // CTAs of the partial FP64 sums

// Device-resident FP64 body state.
struct Body {
  double X[3], U[3], om[3];  // centre, velocity, angular velocity
  double R[9];               // orientation (body frame -> lab), row major
  double P[3], L[3];         // fluid momentum and angular momentum inside the body, previous step
  double Fib[3], Tib[3];     // force and torque the markers put on the fluid, previous step
  int win[6];                // cells holding the IB force (i0, j0, k0, wi, wj, wk); wi = 0: none
  int have_prev;
  int pad;
};

// The current update's geometry, written by its set-up kernel and read by
// the rest: window box, stencil-origin bin box, and whether to go on.
struct Plan {
  int win[6];        // i0, j0, k0, WX, WY, WZ
  int olo[3], on[3]; // first stencil origin and bins per axis
  int W, NB, ok;
  int pad;
};

// One coupled sphere after a fluid step: the buffers of the state that step
// wrote and the body's own arrays.
struct Job {
  const void *f, *g;  // populations of the state [19][N], [7][N] in its storage type
  const void *r;      // 16-bit storage: the state's reference planes [5][N]
  int store;          // IPCU_STORE_*
  float inv_scale;    // 16-bit storage: 1 / the deviations' scale
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
  // global scratch (L2-resident)
  Plan *plan;
  int *morg;               // [nl][3] stencil origins
  float *mw;               // [nl][12] Peskin weights along x, y, z
  float *mub, *mft, *mdf;  // [nl][3] body velocity at the marker, summed force, this iteration's force
  int *bstart, *blist;     // [kMaxBins + 1], [nl] markers by stencil-origin bin, in index order
  float *wu, *wf, *wj;     // [3][kMaxWin] velocity u*, accumulated force density, momentum c j per window cell
  float *wh, *wv;          // [kMaxWin] dt / 2 rho and cell volume
  int *ccnt;               // [kMaxWin] contributions per window cell
  int *clist;              // [kMaxWin][kSlots] its contributions (marker << 6 | node)
  double *part;            // [kParts][12] partial FP64 sums
  unsigned *status;
};

int launch(const Job &j, cudaStream_t s);
int prepare();

}  // namespace ib3d
}  // namespace ipcu
