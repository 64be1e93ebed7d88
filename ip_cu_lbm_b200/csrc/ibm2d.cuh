// Moving immersed boundaries coupled to the fused 2-D solver (ibm2d.cu):
// rigid bodies (one CTA each), Lagrangian markers on their outlines, multi-direct
// forcing with the reference's 4-point Peskin kernel (ref: function/ibm.cu:
// 61-66 weightFunction) and an FP64 rigid-body update built on the
// reference's update_IBbody / update_IBpoint (ref: function/ibm.cu:367-447).
#pragma once
#include <stdint.h>

#include "fused2d.cuh"

namespace ipcu {
namespace ib2d {

constexpr int kThreads = 512;
constexpr int kMaxMarkers = 512;
constexpr int kMaxWindow = 12288;  // cells of the footprint window (old + new stencils)
constexpr int kMaxSlots = 3072;    // distinct cells the stencils touch
constexpr int kHalo = 4;           // a forced cell flags every tile whose halo may reach it

// Device-resident FP64 body state.
struct Body {
  double X[2], U[2], th, om;  // centre, velocity, angle, angular velocity
  double P[2], L;             // fluid momentum and angular momentum inside the body, previous step
  double Fib[2], Tib;         // force and torque (about the centre) the markers put on the fluid, previous step
  int have_prev;              // a coupled step has run: the fields above and the old footprint are valid
  int have_prev2;             // two have: the footprint of two steps back is valid
};

// One coupled body: the fluid's buffers come from the simulation's
// parameter block, the rest is per body.
struct Job {
  f2d::Params fp;  // fluid parameters of the simulation (cur = buffer parity before the step)
  Body *body;
  const double *X0;  // [nl][2] marker positions in the body frame
  const double *dS;  // [nl] arc length per marker
  int *org;          // [nl][2] stencil origin of the previous step's markers
  int *org2;         // [nl][2] ... and of the step before
  float *fext;       // [2][N] force density on the fluid, shared by the simulation's bodies (also fp.fext)
  float *fmark;      // [nl][2] force each marker put on the fluid in the last update (F_l dS_l)
  uint8_t *flag;     // [tiles] this body's slice of fp.ibflag
  int nl, iters;
  double m, I, rho_s, rho_f, grav;  // mass, moment of inertia, densities, gravity (-z)
  double semi_a, semi_b;            // ellipse semi-axes in the body frame (inside test)
  double dz, dt;
};

// Bytes of dynamic shared memory the kernel uses.
size_t smem_bytes();
// Sets the kernel attributes (once per device, outside capture).
int prepare();
// One coupled update after the fluid step that read buffer (j.fp.cur ^ parity).
int launch(const Job &j, int parity, int storage, int qs, cudaStream_t s);
// The same for njobs bodies (device array), one CTA each.
int launch_batched(const Job *jobs, int njobs, int parity, int storage, int qs, cudaStream_t s);

}  // namespace ib2d
}  // namespace ipcu
