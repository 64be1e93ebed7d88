/*
 * ipcu_sim3d.h -- 3-D structured solver of libipcu (included by ipcu.h).
 *
 * One simulation = one box of nx x ny x nz cells on a uniform lattice (or
 * with stretched x and y axes, ipcu_sim3d_create_stretched):
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
 *
 * 16-bit storage (storage IPCU_STORE_F16 / IPCU_STORE_BF16; collision,
 * streaming and forcing stay FP32): each cell keeps five reference values
 * r [5][N] (p, u_x/c, u_y/c, u_z/c, S: what its collision formed in the step
 * that wrote it) in the storage type, and its populations as deviations
 * from the linear equilibria of that reference,
 * f_k - w_k (p + 3 e_k.u) and g_k - w_k S (1 + 4 e_k.u), scaled by 2^12
 * (FP16) or 1 (BF16): 148 B per cell and step against 232 B. Every box,
 * uniform or stretched, runs the flux-form kernel (stencil 3 unless the
 * axes say otherwise). Status bit 2: a stored magnitude beyond the format's
 * range. Raw transfer (upload/download) of f and g is FP32-only.
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
  int32_t storage;      /* IPCU_STORE_* (16-bit: see below) */
  int32_t pad;
} ipcu_sim3d_config;

typedef struct ipcu_sim3d ipcu_sim3d;

/* Creates a simulation at rest (f = 0, g = w_k S0, F = 0); s0: host, N
 * values x fastest (NULL = 0). */
int ipcu_sim3d_create(const ipcu_sim3d_config *cfg, const double *s0, ipcu_stream_t stream, ipcu_sim3d **out);

/* Stretched x and y axes (z stays uniform): cell centres and widths per
 * axis (host arrays; NULL keeps that axis uniform; every width >= dz), and
 * the interpolation stencil of the reference's conservative flux form
 * (ref: function/adv.cu:50-257): 3 (quadratic, two upstream nodes and one
 * downstream) or 5 (the reference's centred 5-point stencil). Populations
 * moving along x or y take the 1-D flux form, those moving along an xy
 * diagonal the corner-transport form of set_out (adv.cu:100-145), z is an
 * exact shift. Ghosts across x and y walls are mirror images of their
 * owners for every quantity the flux form reads; sources outside the box
 * bounce back. */
typedef struct ipcu_sim3d_axes {
  const double *x, *wx; /* nx cell centres and widths along x */
  const double *y, *wy; /* ny cell centres and widths along y */
  int32_t ns;           /* 3 or 5 */
} ipcu_sim3d_axes;
int ipcu_sim3d_create_stretched(const ipcu_sim3d_config *cfg, const ipcu_sim3d_axes *axes, const double *s0,
                                ipcu_stream_t stream, ipcu_sim3d **out);
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
/* Raw FP32 state transfer, asynchronous (pinned host buffers): f, g, F.
 * With 16-bit storage only F (IPCU_ERR_UNSUPPORTED for f or g). */
int ipcu_sim3d_upload(ipcu_sim3d *sim, const float *f, const float *g, const float *F);
int ipcu_sim3d_download(ipcu_sim3d *sim, float *f, float *g, float *F);
/* S, u_x, u_y, u_z of every cell ([4][N] FP32, the values ipcu_sim3d_get
 * serves) formed on the device and copied into `out` (pinned host or device
 * memory), asynchronous on the simulation's stream. */
int ipcu_sim3d_macro_async(ipcu_sim3d *sim, float *out);
int ipcu_sim3d_sync(ipcu_sim3d *sim);
/* Sticky error flags (bit 0: non-finite moment seen). Synchronises. */
int ipcu_sim3d_status(ipcu_sim3d *sim, uint32_t *flags);
int64_t ipcu_sim3d_cells(const ipcu_sim3d *sim);
/* Algorithmic bytes per cell and step: f, g, F (16-bit: and the reference
 * planes) each read and written once. */
int64_t ipcu_sim3d_bytes_per_cell(const ipcu_sim3d *sim);
/* Versioned binary snapshot (configuration, axes, stencil, step count, raw
 * state in its storage type) and its restore into a new simulation; a
 * restored run continues bit-identically. */
int ipcu_sim3d_save(ipcu_sim3d *sim, const char *path);
int ipcu_sim3d_load(const char *path, ipcu_stream_t stream, ipcu_sim3d **out);
/* Moving rigid sphere (one per simulation; the sphere of the reference's
 * SphereFallSuzuki2018 driver): markers on its surface (body frame, [n][3],
 * n <= 1024) carry areas dA; each step, after the fluid step, multi-direct
 * forcing with the reference's 4-point Peskin kernel per axis (ref:
 * function/ibm.cu:61-66 weightFunction; on stretched x and y axes the kernel
 * is evaluated in cell-index space) makes the fluid follow the body at the
 * markers, the force density enters the next fluid step, and the body moves
 * by an FP64 momentum balance built on the reference's update_IBbody /
 * update_IBpoint (ref: function/ibm.cu:367-447) in three dimensions:
 * reaction of the IB force, buoyancy -(1 - rho_f/rho_s) m gravity along z,
 * the change of the fluid momentum inside the sphere. Drops recorded
 * graphs; snapshots of a simulation with a sphere are refused
 * (IPCU_ERR_UNSUPPORTED). Status bit 8: the footprint outgrew the update's
 * window (the update was skipped). */
typedef struct ipcu_ib_sphere3d {
  double xc, yc, zc;  /* centre (physical units; cell centres at the axes' x, y and (k + 1/2) dz) */
  double u, v, w;     /* initial velocity */
  double radius;
  double rho_s, rho_f; /* sphere and fluid density */
  double gravity;
  int32_t iters;      /* multi-direct forcing iterations (3) */
  int32_t pad;
} ipcu_ib_sphere3d;
int ipcu_sim3d_ib_attach(ipcu_sim3d *sim, const ipcu_ib_sphere3d *body, const double *markers, const double *dA,
                         int32_t n);
/* Sphere state: centre (3), velocity (3), angular velocity (3), and the IB
 * force (3) and torque (3) the markers put on the fluid in the last step
 * (15 values). Synchronises. */
int ipcu_sim3d_ib_body(ipcu_sim3d *sim, double *out);
int64_t ipcu_sim3d_steps(const ipcu_sim3d *sim);

#endif /* IPCU_SIM3D_H */
