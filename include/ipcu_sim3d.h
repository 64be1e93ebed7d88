/*
 * ipcu_sim3d.h -- 3-D structured solver of libipcu (included by ipcu.h).
 *
 * One simulation = one box of nx x ny x nz cells on a uniform lattice:
 * D3Q19 flow (MRT with the d'Humieres moment basis, the five shear moments
 * relaxing with 1/tau and all others with rate 1, as the reference's
 * unit-rate S file; or BGK) and a D3Q7 passive salinity with the
 * regularised collision, Boussinesq buoyancy -g_bouss S along z and the
 * pressure-gradient force, halfway bounce-back on all six faces. Each step
 * is the reference's LockExchange step order (ref: LockExchange/
 * LockExchange.cu:220-236; function/collision.cu:3-188,238-257) on the
 * D3Q19 / D3Q7 subsets of its D3Q27 velocity order (ref: function/
 * basic.cu:88-97), fused into one kernel launch.
 *
 * Storage: FP32 structure-of-arrays, x fastest, then y, then z: f [19][N],
 * g [7][N] and the previous step's force F [3][N]; ping-pong buffers
 * resident in HBM. D3Q7 weights 1/4, 1/8 (cs^2 = 1/4), equilibrium
 * w_k S (1 + 4 e_k.u/c). The reference has no D3Q19/D3Q7 path: this mode
 * has no reference counterpart beyond the shared kernel rules.
 */
#ifndef IPCU_SIM3D_H
#define IPCU_SIM3D_H
#include <stdint.h>

typedef struct ipcu_sim3d_config {
  int32_t nx, ny, nz;
  int32_t mrt;          /* 1 MRT (unit non-shear rates), 0 BGK */
  double dz, dt;        /* lattice spacing and time step, c = dz/dt */
  double tau, taus;     /* relaxation times of f and of the salinity */
  double rho0, rho_sal; /* rho = rho0 + rho_sal S */
  double g_bouss;       /* buoyancy -g_bouss S along z */
} ipcu_sim3d_config;

typedef struct ipcu_sim3d ipcu_sim3d;

/* Creates a simulation at rest (f = 0, g = w_k S0, F = 0); s0: host, N
 * values x fastest (NULL = 0). */
int ipcu_sim3d_create(const ipcu_sim3d_config *cfg, const double *s0, ipcu_stream_t stream, ipcu_sim3d **out);
void ipcu_sim3d_destroy(ipcu_sim3d *sim);
/* Advances nsteps (asynchronous on the simulation's stream). */
int ipcu_sim3d_step(ipcu_sim3d *sim, int64_t nsteps);
/* The same steps replayed from a CUDA graph of two steps. */
int ipcu_sim3d_step_graph(ipcu_sim3d *sim, int64_t nsteps);
/* Fields: "f" (19 N), "g" (7 N), "F" (3 N), "S", "p", "ux", "uy", "uz" (N).
 * Host FP64 output; u includes F dt / 2 rho. Synchronises. */
int ipcu_sim3d_get(ipcu_sim3d *sim, const char *field, double *out, int64_t n);
/* Overwrites f (19 N), g (7 N), F (3 N) from host FP64 arrays (NULL keeps). */
int ipcu_sim3d_set_state(ipcu_sim3d *sim, const double *f, const double *g, const double *F);
/* Raw FP32 state transfer, asynchronous (pinned host buffers): f, g, F. */
int ipcu_sim3d_upload(ipcu_sim3d *sim, const float *f, const float *g, const float *F);
int ipcu_sim3d_download(ipcu_sim3d *sim, float *f, float *g, float *F);
int ipcu_sim3d_sync(ipcu_sim3d *sim);
/* Sticky error flags (bit 0: non-finite moment seen). Synchronises. */
int ipcu_sim3d_status(ipcu_sim3d *sim, uint32_t *flags);
int64_t ipcu_sim3d_cells(const ipcu_sim3d *sim);
/* Algorithmic bytes per cell and step: f, g, F each read and written once. */
int64_t ipcu_sim3d_bytes_per_cell(const ipcu_sim3d *sim);

#endif /* IPCU_SIM3D_H */
