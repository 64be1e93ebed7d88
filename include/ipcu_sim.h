/*
 * ipcu_sim.h -- structured-grid solver of libipcu (included by ipcu.h).
 *
 * One simulation = one rectangular box of nx x nz cells (2-D, x-z plane,
 * D2Q9 flow) with a scalar lattice (D2Q5 or the reference's Q9 scalar),
 * rectilinear coordinates and one interpolated axis. The scalar is either
 *   - salinity (IPCU_SCALAR_SALINITY): each step is the reference's
 *     LockExchange step (ref: LockExchange/LockExchange.cu:220-236 without
 *     the wall model): equilibrium, Boussinesq force, MRT/SRT collision,
 *     conservative interpolated streaming of f, regularised scalar
 *     collision and streaming of g, then the moments; or
 *   - the Allen-Cahn phase field (IPCU_SCALAR_PHASE): the reference's
 *     two-phase step (ref: RTinstability/RTinstability.cu:177-206):
 *     rho = rhoL + (rhoH - rhoL) phi, surface tension and the mixture's
 *     weight in the force, the conservative Allen-Cahn collision with its
 *     d(phi u)/dt term (function/collision.cu:57-113,190-223);
 * fused into one kernel launch that reads each stored value once and
 * writes it once.
 *
 * Storage: structure-of-arrays, x fastest, ping-pong buffers resident in
 * HBM; distributions in FP32 or in FP16/BF16 (the pressure-form f is a
 * deviation; g is stored shifted by w_k*S_ref), macroscopic S, u_x, u_z in
 * FP32. Counts are exact int64.
 */
#ifndef IPCU_SIM_H
#define IPCU_SIM_H
#include <stdint.h>

/* grid kinds for the interpolated streaming */
#define IPCU_GEO_UNIFORM 0 /* exact shift */
#define IPCU_GEO_X5 1      /* x nonuniform, 5-point Lagrange flux form (reference scheme) */
#define IPCU_GEO_X3 2      /* x nonuniform, 3-point upwind-biased quadratic flux form */
#define IPCU_GEO_Z5 3      /* z nonuniform, 5-point */
#define IPCU_GEO_Z3 4      /* z nonuniform, 3-point quadratic upwind */

#define IPCU_STORE_F32 0
#define IPCU_STORE_F16 1
#define IPCU_STORE_BF16 2

#define IPCU_WALL_SLIP 0 /* specular reflection, reference set_bound2D tables */
#define IPCU_WALL_BB 1   /* halfway bounce-back */

#define IPCU_SCALAR_SALINITY 0 /* passive salinity, Boussinesq buoyancy */
#define IPCU_SCALAR_PHASE 1    /* conservative Allen-Cahn phase field, two-phase density */

typedef struct ipcu_sim_config {
  int32_t nx, nz;       /* cells */
  int32_t q_scalar;     /* 0 none, 5 D2Q5, 9 reference Q9 scalar */
  int32_t geometry;     /* IPCU_GEO_* */
  int32_t storage;      /* IPCU_STORE_* */
  int32_t wall;         /* IPCU_WALL_* on all four walls */
  int32_t mrt;          /* 1 MRT (matrices below), 0 SRT */
  int32_t scalar_kind;  /* IPCU_SCALAR_* (phase field needs q_scalar 5 or 9) */
  double dz;            /* lattice spacing; c = dz/dt */
  double dt;
  const double *x;      /* host, nx cell centres (NULL: (i+0.5)*dz) */
  const double *z;      /* host, nz cell centres (NULL: (l+0.5)*dz) */
  const double *wx;     /* host, nx cell widths (NULL: dz) */
  const double *wz;     /* host, nz cell widths (NULL: dz) */
  double tau, taus;     /* relaxation times of f and g (phase field: tau_phi; the reference fixes 0.58) */
  double rhoL, rhoH, phi; /* salinity: rho = rhoL + (rhoH-rhoL)*phi + rho_sal*S; phase field:
                             rho = rhoL + (rhoH-rhoL)*phi(x) with phi the scalar field */
  double rho_sal;       /* reference: 0.824493 */
  double g_bouss;       /* buoyancy Fz = -g_bouss*S (reference: 0.824493*9.81) */
  double s_ref;         /* unused (16-bit storage keeps deviations from the local equilibrium) */
  const double *M;      /* host 9x9 moment matrix (row-major), MRT only */
  const double *Minv;   /* host 9x9 inverse */
  const double *S;      /* host 9 relaxation rates (shear entries 7,8 are replaced by 1/tau) */
  /* phase field only */
  double sigma;         /* surface tension */
  double pf_width;      /* interface thickness W (reference: items PFthick) */
  double gravity;       /* weight -rho*gravity along z (reference: 9.81) */
} ipcu_sim_config;

typedef struct ipcu_sim ipcu_sim;

/* Creates a simulation on the current device and stream. Initial state:
 * f = equilibrium of p*=0, u=0 (zero), g = equilibrium of S, S given per
 * cell in s0 (host, nx*nz, x fastest; NULL = 0). Returns a status. */
int ipcu_sim_create(const ipcu_sim_config *cfg, const double *s0, ipcu_stream_t stream, ipcu_sim **out);
void ipcu_sim_destroy(ipcu_sim *sim);
/* Advances nsteps (asynchronous on the sim's stream). */
int ipcu_sim_step(ipcu_sim *sim, int64_t nsteps);
/* Same steps recorded once into a CUDA graph of `chunk` steps and replayed. */
int ipcu_sim_step_graph(ipcu_sim *sim, int64_t nsteps, int32_t chunk);
/* Field names: "f" (9*N), "g" (q_scalar*N), "S", "ux", "uz", "p", "rho"
 * (N each). Host output in FP64, x fastest, population-major for f/g.
 * Synchronises the sim's stream. */
int ipcu_sim_get(ipcu_sim *sim, const char *field, double *host_out, int64_t n);
/* Overwrites the state from host FP64 arrays (f: 9*N, g: q*N, S/ux/uz: N). */
int ipcu_sim_set_state(ipcu_sim *sim, const double *f, const double *g, const double *S, const double *ux,
                       const double *uz);
/* Sticky error flags (bit 0: non-finite moment seen). Synchronises. */
int ipcu_sim_status(ipcu_sim *sim, uint32_t *flags);
/* Raw state transfer in the storage layout, asynchronous on the sim's
 * stream (host buffers should be pinned): f (9*N values of the storage
 * type, already scaled), g (q_scalar*N, scaled and shifted), mac (FP32
 * [3][N]: S, u_x, u_z). NULL skips a buffer. */
int ipcu_sim_upload(ipcu_sim *sim, const void *f, const void *g, const float *mac);
int ipcu_sim_download(ipcu_sim *sim, void *f, void *g, float *mac);
int ipcu_sim_sync(ipcu_sim *sim);
/* FP64 area-weighted totals of p* (sum of the 9 FP32 populations f[k*N+i])
 * and of S (mac[i]) with cell weights wx[x]*wz[z], written to out[0..1]
 * (all device pointers), without allocating anything. No counterpart in the
 * reference: it exists for callers that cannot allocate device memory where
 * they need the check -- hosts that give all device memory to their own
 * pool, loops that must not enter the driver's allocator. Its scratch is a
 * fixed file-scope device array, so it accepts at most 16,777,216 cells
 * (IPCU_ERR_CAPACITY beyond); the first call on a device resolves that
 * array's address (make it before any capture, with the stream's device
 * current); concurrent calls race on the shared array. FP32 populations
 * only (16-bit storage keeps p* in its own plane: use ipcu_sim_totals).
 * The result equals ipcu_sim_totals' to rounding, not bit for bit (more
 * blocks, another FP64 summation order). */
int ipcu_totals_noalloc_f32(const float *f, const float *mac, const float *wx, const float *wz, int nx, int nz,
                            double *out, ipcu_stream_t stream);
/* Time steps taken since creation or restore. */
int64_t ipcu_sim_steps(const ipcu_sim *sim);
/* Versioned binary snapshot (configuration, geometry, MRT matrices, step
 * count, raw state, and the attached moving bodies: their descriptions
 * and device state) and its restore into a new simulation; a restored run
 * continues bit-identically (replaces basic.cu:31-56 save_status). Version
 * 5; versions 3 and 4 (at most one body) still load. */
int ipcu_sim_save(ipcu_sim *sim, const char *path);
int ipcu_sim_load(const char *path, ipcu_stream_t stream, ipcu_sim **out);
/* Field CSV in the reference's column order and cell order (basic.cu:16-28). */
int ipcu_sim_write_csv(ipcu_sim *sim, const char *path);
/* Bytes of one stored distribution value (4 FP32, 2 FP16/BF16). */
int32_t ipcu_sim_storage_bytes(const ipcu_sim *sim);
int64_t ipcu_sim_cells(const ipcu_sim *sim);
/* Device pointers of the current state buffers (for zero-copy consumers). */
int ipcu_sim_device_state(ipcu_sim *sim, void **f, void **g, float **mac);
/* Bytes each stored value moves per cell and step (algorithmic traffic). */
int64_t ipcu_sim_bytes_per_cell(const ipcu_sim *sim);
/* FP64 domain sums of S and p* weighted by cell area (dx*dz/dz^2), the
 * reference's conservation diagnostic (ref: function/basic.cu:9-15). */
int ipcu_sim_totals(ipcu_sim *sim, double *sum_p, double *sum_s);
/* Lean flow-only step (on by default where allowed: FP32 storage, nx % 4 ==
 * 0, no scalar lattice, uniform S). The step kernel then moves the nine
 * populations only: the constant S plane is neither read nor written, and
 * the velocity planes are stored only in tiles where an immersed body's
 * force acted; elsewhere the velocity is recomputed from the populations,
 * bit for bit the value the full step stores (ref: the update_rho moments,
 * function/collision.cu:238-257). Field reads, downloads and snapshots
 * complete the planes first. Uploading a non-uniform S plane turns it off.
 * ipcu_sim_set_lean(sim, 0) forces the full step (IPCU_ERR_UNSUPPORTED when
 * enabling a configuration that does not allow it); ipcu_sim_lean reports
 * whether it is on. */
int ipcu_sim_set_lean(ipcu_sim *sim, int enable);
int ipcu_sim_lean(const ipcu_sim *sim);
/* Push form of the lean step (on by default where allowed: bounce-back
 * walls, uniform grid, two-moment MRT): each cell collides in registers and
 * pushes its populations to the cells they stream into, no halo, no shared
 * memory; a tile that applied a body force records that force instead of
 * the velocity (the velocity stays recomputable bit for bit). Results equal
 * the tile kernel's bit for bit. ipcu_sim_set_push(sim, 0) selects the
 * tile form of the lean step (IPCU_ERR_UNSUPPORTED when enabling where not
 * allowed); ipcu_sim_push reports whether the push form is selected. */
int ipcu_sim_set_push(ipcu_sim *sim, int enable);
int ipcu_sim_push(const ipcu_sim *sim);

/* Batched stepping of many resident simulations (continuous-batching
 * serving): each call advances every listed simulation by nsteps with one
 * launch per step per kernel class (storage, scalar lattice, geometry); CTAs
 * walk a device work list of (simulation, tile). A simulation's arithmetic is
 * the same tile by tile as when it runs alone. Synchronous; the batch
 * stream first waits (on the device) for work already queued on each
 * simulation's own stream. */
typedef struct ipcu_batch ipcu_batch;
int ipcu_batch_create(ipcu_stream_t stream, ipcu_batch **out);
void ipcu_batch_destroy(ipcu_batch *batch);
int ipcu_batch_step(ipcu_batch *batch, ipcu_sim *const *sims, int n, int64_t nsteps);
/* The same steps enqueued without waiting: each listed simulation's own
 * stream is ordered after them, so its reads, further steps and destruction
 * see the results; ipcu_batch_sync waits for everything enqueued. A server
 * admits new requests on the host while the GPU runs the batch. */
int ipcu_batch_launch(ipcu_batch *batch, ipcu_sim *const *sims, int n, int64_t nsteps);
/* The same with a step count per simulation (nsteps[i] >= 0; 0 leaves it
 * out): the simulations still stepping at each step share one launch per
 * kernel class, so a server advances every admitted request to its own end
 * of the tick with one call. */
int ipcu_batch_launch_each(ipcu_batch *batch, ipcu_sim *const *sims, const int64_t *nsteps, int n);
int ipcu_batch_sync(ipcu_batch *batch);
/* Progress marks: ipcu_batch_mark records the point reached by everything
 * enqueued so far and returns its handle (a ring of 4); ipcu_batch_wait_mark
 * waits for it. A server keeps the host one tick ahead of the GPU with them. */
int ipcu_batch_mark(ipcu_batch *batch);
int ipcu_batch_wait_mark(ipcu_batch *batch, int mark);
/* Graph mode (enable 1): each launch call's kernel sequence is captured into
 * one CUDA graph and replayed, the executable graph updated in place while
 * the sequence keeps its shape (IPCU_ERR_UNSUPPORTED on the legacy default
 * stream). ipcu_batch_graph_stats: in-place updates and instantiations so far. */
int ipcu_batch_set_graph(ipcu_batch *batch, int enable);
int ipcu_batch_graph_stats(const ipcu_batch *batch, int64_t *updates, int64_t *instantiations);
/* CTAs per SM of the batched grid for one kernel class (storage, scalar
 * lattice, geometry, scalar kind); 0 restores the default (4). The
 * autotuner of the serving loop sets it. */
int ipcu_batch_set_ctas(ipcu_batch *batch, int storage, int q_scalar, int geometry, int scalar_kind, int ctas_per_sm);
/* Moving immersed boundaries: up to 16 rigid bodies per simulation, as the
 * reference's IB_index loop over bodies (ref: function/ibm.cu:367-424)
 * (uniform lattice, salinity or no scalar). Markers on the outline (body frame,
 * physical units) carry arc lengths dS; each step, after the fluid step,
 * multi-direct forcing with the reference's 4-point Peskin kernel
 * (ref: function/ibm.cu:61-66 weightFunction) makes the fluid follow the
 * body at the markers, the force density enters the next fluid step, and
 * the body moves by an FP64 momentum balance built on the reference's
 * update_IBbody / update_IBpoint (ref: function/ibm.cu:367-447): the
 * reaction of the IB force, buoyancy -(1 - rho_f/rho_s) m gravity along z
 * and the change of the fluid momentum inside the body. No counterpart of
 * the reference's own IB coupling (get_IBMGw2), which stays available
 * through the kernel-entry API above. The coupling is stable at density
 * ratios down to about one for bodies at least 4 cells thick (semi-axes
 * >= 4 dz): a thinner body lies wholly inside its own 4-point stencils and
 * its interior fluid no longer follows it. Bodies share the force density
 * and are updated side by side: they must stay apart (no contact model, as
 * in the reference); a body attached closer than 6 cells (outline to
 * outline, the outlines taken as circles of the largest marker radius) to
 * another is refused with IPCU_ERR_ARG. */
typedef struct ipcu_ib_body2d {
  double xc, zc, theta;   /* centre (cell centres at (i + 1/2) dz) and angle */
  double u, w, omega;     /* initial velocity and angular velocity */
  double rho_s, rho_f;    /* body and fluid density */
  double area, inertia;   /* area and polar second moment of area (integral of r^2 dA) */
  double semi_a, semi_b;  /* ellipse semi-axes (body frame x, z): cells whose centre lies inside
                             carry the fluid momentum the body update adds back */
  double gravity;
  int32_t iters;          /* multi-direct forcing iterations (3) */
  int32_t pad;
} ipcu_ib_body2d;
/* Attaches one more body (n <= 512 markers, [n][2] x, z; it gets the next
 * index, from 0); IPCU_ERR_UNSUPPORTED for stretched geometries and the
 * phase field, IPCU_ERR_CAPACITY past 16 bodies. Drops recorded graphs.
 * Status bit 8: a body's stencils outgrew the kernel's window (its update
 * was skipped). */
int ipcu_sim_ib_attach(ipcu_sim *sim, const ipcu_ib_body2d *body, const double *markers, const double *dS, int32_t n);
/* Bodies attached. */
int32_t ipcu_sim_ib_count(const ipcu_sim *sim);
/* Markers of body `index`, 9 values each (x, y, z, u, v, w, Fx, Fy, Fz:
 * position and velocity now, and the force the marker put on the fluid in
 * the last update; y = dz/2), cap >= the marker count; returns the marker
 * count (a negative status on error). ipcu_sim_ib_markers is body 0. The
 * CSV holds every body's markers, body after body, in the reference's
 * IB_csv column order, header "x,y,z,velx,vely,velz,ax,ay,az" (ref:
 * function/ibm.cu:3-14). */
int32_t ipcu_sim_ib_markers_at(ipcu_sim *sim, int32_t index, double *out, int32_t cap);
int32_t ipcu_sim_ib_markers(ipcu_sim *sim, double *out, int32_t cap);
int ipcu_sim_write_ib_csv(ipcu_sim *sim, const char *path);
/* State of body `index`: x, z, u, w, theta, omega and the IB force (x, z)
 * and torque the markers put on the fluid in the last step (9 values).
 * Synchronises. ipcu_sim_ib_body is body 0. ipcu_sim_get serves the force
 * density of all bodies as fields "ibfx", "ibfz". */
int ipcu_sim_ib_body_at(ipcu_sim *sim, int32_t index, double *out);
int ipcu_sim_ib_body(ipcu_sim *sim, double *out);
/* A new non-blocking CUDA stream (it does not synchronise with the legacy
 * default stream) and its release; work still queued on a released stream
 * completes. A server gives each admitted simulation one, so that a
 * simulation's set-up never waits for the batch in flight. */
int ipcu_stream_create(ipcu_stream_t *out);
int ipcu_stream_destroy(ipcu_stream_t stream);
/* Device bytes a simulation holds (state, ping-pong, tables). */
int64_t ipcu_sim_device_bytes(const ipcu_sim *sim);

#endif /* IPCU_SIM_H */
