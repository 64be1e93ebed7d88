/*
 * ipcu.h -- C ABI of libipcu, the B200 (sm_100a) implementation of the
 * IP_CU_LBM per-step lattice Boltzmann path.
 *
 * Two surfaces:
 *   1. Reference-compatible kernel entries. One launcher per kernel of the
 *      reference library (Kasahara1341/IP_CU_LBM function/*.cu, declared in
 *      all.hpp:38-158), same name with an ipcu_ prefix and a _f32/_f64
 *      suffix, same argument order, same array-of-structures buffers
 *      f[cell*Q+k] over the compacted cell list and the same float/double
 *      items[] parameter block (itemIndex.hpp:4-33). Two trailing arguments
 *      replace the reference's <<<numBlocks, blockSize>>>: `nthreads`
 *      (numBlocks*blockSize; <= 0 lets the launcher pick a persistent grid,
 *      the kernels are grid-stride) and the CUDA stream (NULL = the legacy
 *      default stream the reference used). Launchers are asynchronous and
 *      return a status (0 = ok); the reference returned nothing and its
 *      drivers polled cudaGetLastError() once per step
 *      (LockExchange/LockExchange.cu:240-244).
 *   2. Structured-grid solver (ipcu_sim_*): fused collide-and-stream kernels
 *      over structure-of-arrays storage, one launch per step, FP32 or
 *      FP16/BF16 shifted storage, with exact int64 cell counts.
 *
 * Every pointer argument of the kernel entries is a device pointer unless
 * the comment says host. No function throws across the ABI.
 */
#ifndef IPCU_H
#define IPCU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *ipcu_stream_t; /* == cudaStream_t */

/* status codes */
#define IPCU_OK 0
#define IPCU_ERR_ARG -1
#define IPCU_ERR_CUDA -2
#define IPCU_ERR_NOMEM -3
#define IPCU_ERR_CAPACITY -4
#define IPCU_ERR_NONFINITE -5
#define IPCU_ERR_UNSUPPORTED -6
#define IPCU_ERR_IO -7
#define IPCU_ERR_TIMEOUT -8

const char *ipcu_status_string(int code);
const char *ipcu_last_cuda_error(void);
int ipcu_version(void);

/* ======================================================================
 * 1. Reference-compatible kernel entries
 * ====================================================================== */
#define IPCU_LEGACY_DECLS(T, S)                                                                                \
  /* collision.cu:3-14 equ_f */                                                                                \
  int ipcu_equ_f_##S(T *items, T *feq, T *pressure, T *velx, T *vely, T *velz, int64_t nthreads,               \
                     ipcu_stream_t stream);                                                                   \
  /* collision.cu:16-27 equ_g */                                                                               \
  int ipcu_equ_g_##S(T *items, T *feq, T *sal, T *velx, T *vely, T *velz, int64_t nthreads,                    \
                     ipcu_stream_t stream);                                                                   \
  /* collision.cu:28-55 wall_function */                                                                       \
  int ipcu_wall_function_##S(T *items, T *delX, T *delY, int x, int y, int z, int wall_number, int *wall,       \
                             T *velx, T *vely, T *velz, T *Fx, T *Fy, T *rho, int64_t nthreads,                \
                             ipcu_stream_t stream);                                                           \
  /* collision.cu:57-112 Force (Boussi_flag: 0/1) */                                                           \
  int ipcu_Force_##S(T *items, int Boussi_flag, int *neib, T *f, T *feq, T *tau, T *Fk, T *Fx, T *Fy, T *Fz,    \
                     T *pressure, T *rho, T *sal, T *phi, T *velx, T *vely, T *velz, T *delX, T *delY,          \
                     T *posx, T *posy, T *posz, int64_t nthreads, ipcu_stream_t stream);                      \
  /* collision.cu:115-150 col_f_MRT (Mconst = MM of set_M) */                                                  \
  int ipcu_col_f_MRT_##S(T *items, T *tau, T *f, T *ftmp, T *feq, T *Fk, T *M, T *M_inv, T *S, T *Mconst,       \
                         int64_t nthreads, ipcu_stream_t stream);                                             \
  /* collision.cu:151-165 col_f_SRT */                                                                         \
  int ipcu_col_f_SRT_##S(T *items, T *tau, T *f, T *ftmp, T *feq, T *Fk, int64_t nthreads,                     \
                         ipcu_stream_t stream);                                                               \
  /* collision.cu:167-188 col_g_reg */                                                                         \
  int ipcu_col_g_reg_##S(T *items, T *taus, T *g, T *gtmp, T *geq, T *sal, T *velx, T *vely, T *velz,           \
                         int64_t nthreads, ipcu_stream_t stream);                                             \
  /* collision.cu:190-223 col_PF */                                                                            \
  int ipcu_col_PF_##S(T *items, int *neib, T *taus, T *g, T *gtmp, T *geq, T *phi, T *velx, T *vely, T *velz,   \
                      T *phiold, T *uold, T *vold, T *wold, T *posx, T *posy, T *posz, int64_t nthreads,        \
                      ipcu_stream_t stream);                                                                  \
  /* collision.cu:225-236 update_scalar */                                                                     \
  int ipcu_update_scalar_##S(T *items, T *g, T *scalar, int64_t nthreads, ipcu_stream_t stream);               \
  /* collision.cu:238-257 update_rho */                                                                        \
  int ipcu_update_rho_##S(T *items, T rhoL, T rhoH, T *f, T *Fx, T *Fy, T *Fz, T *pressure, T *sal, T *phi,     \
                          T *rho, T *velx, T *vely, T *velz, int64_t nthreads, ipcu_stream_t stream);         \
  /* collision.cu:258-264 resetF */                                                                            \
  int ipcu_resetF_##S(T *items, T *Fx, T *Fy, T *Fz, int num_F, int64_t nthreads, ipcu_stream_t stream);       \
  /* adv.cu:3-13 set_wall_f */                                                                                 \
  int ipcu_set_wall_f_##S(T *items, int *neib, T *f, int64_t nthreads, ipcu_stream_t stream);                  \
  /* adv.cu:50-147 set_out */                                                                                  \
  int ipcu_set_out_##S(T *items, int *neib, T *ftmp, T *fout, T *fin, T *finy, T *posx, T *posy, T *delX,       \
                       T *delY, int64_t nthreads, ipcu_stream_t stream);                                      \
  /* adv.cu:148-175 set_fin */                                                                                 \
  int ipcu_set_fin_##S(T *items, int *neib, int *nextK, T *fin, T *finy, int64_t nthreads, ipcu_stream_t stream); \
  /* adv.cu:176-187 reset_f */                                                                                 \
  int ipcu_reset_f_##S(T *items, T *ftmp, T *fin, T *f, int64_t nthreads, ipcu_stream_t stream);               \
  /* adv.cu:188-232 set_wall_f_inv */                                                                          \
  int ipcu_set_wall_f_inv_##S(T *items, int *neib, int *nextB, int *nextK, T *f, int64_t nthreads,              \
                              ipcu_stream_t stream);                                                          \
  /* adv.cu:234-244 set_tmp */                                                                                 \
  int ipcu_set_tmp_##S(T *items, int *neib, T *f, T *ftmp, T *fout, T *fin, int64_t nthreads,                  \
                       ipcu_stream_t stream);                                                                 \
  /* adv.cu:245-257 IP_process (slip: 0 specular slip, 1 bounce-back) */                                       \
  int ipcu_IP_process_##S(T *d_items, int numBlocks, int blockSize, int *d_neib, T *d_f, T *d_feq, T *d_ftmp,   \
                          T *d_fout, int *d_nextB, int *d_nextK, T *d_posx, T *d_posy, T *d_delX, T *d_delY,   \
                          int slip, ipcu_stream_t stream);                                                    \
  /* set_bound.cu:164-183 set_wall_propagation */                                                              \
  int ipcu_set_wall_propagation_##S(T *items, int boundary_condition, int *neib, int *nextK, int *nextB,        \
                                    T *ftmp, int64_t nthreads, ipcu_stream_t stream);                         \
  /* propagation.cu:2-12 propagation */                                                                        \
  int ipcu_propagation_##S(T *items, int *neib, T *f, T *ftmp, int64_t nthreads, ipcu_stream_t stream);        \
  /* basic.cu:274-284 reset_wall_fin */                                                                        \
  int ipcu_reset_wall_fin_##S(T *items, T *fin, T *finy, int64_t nthreads, ipcu_stream_t stream);              \
  /* basic.cu:254-261 set_wall_rho */                                                                          \
  int ipcu_set_wall_rho_##S(T *items, int *neib, T *rho, int64_t nthreads, ipcu_stream_t stream);              \
  /* basic.cu:262-273 reset_pressure */                                                                        \
  int ipcu_reset_pressure_##S(T *items, T *pressure, T *f, T *velx, T *vely, T *velz, T alpha,                  \
                              int64_t nthreads, ipcu_stream_t stream);                                        \
  /* basic.cu:285-339 LES */                                                                                   \
  int ipcu_LES_##S(T *items, int *neib, T *tau, T *taus, T *phi, T *rho, T muL, T muH, T *velx, T *vely,        \
                   T *velz, T *posx, T *posy, T *posz, int64_t nthreads, ipcu_stream_t stream);               \
  /* ibm.cu:124-274 get_IBMGw2 */                                                                              \
  int ipcu_get_IBMGw2_##S(T *items, int *lattice_id, int *neib, T *f, T *tau, T *posx, T *posy, T *posz,        \
                          T *posw, T *posB, T *nBvec, T *velx, T *vely, T *velz, T *velw, T *Fx, T *Fy, T *Fz,  \
                          T *Gw, T rhof, int64_t nthreads, ipcu_stream_t stream);                             \
  /* ibm.cu:346-365 update_velIBM */                                                                           \
  int ipcu_update_velIBM_##S(T *items, int *lattice_id, T *f, T *ftmp, T *pressure, T *tau, T *velx, T *vely,   \
                             T *velz, T *velx_old, T *vely_old, T *velz_old, T *Fx, T *Fy, T *Fz,              \
                             int64_t nthreads, ipcu_stream_t stream);                                         \
  /* ibm.cu:367-424 update_IBbody */                                                                           \
  int ipcu_update_IBbody_##S(T *items, int IB_index, T *massB, T *densB, T *inertia, T *FB, T *posB, T *Torque, \
                             T *velB, T *quat, T *quaS, T *angleVB, T *posw, T *Gw, T *quatold, T rhof,        \
                             int64_t nthreads, ipcu_stream_t stream);                                         \
  /* ibm.cu:426-447 update_IBpoint */                                                                          \
  int ipcu_update_IBpoint_##S(T *items, int IB_index, T *posB, T *velB, T *angleVB, T *quaS, T *posw,           \
                              T *oposw, T *nBvec, T *onBvec, T *velw, int64_t nthreads, ipcu_stream_t stream); \
  /* ibm.cu:449-463 search_IBlattice */                                                                        \
  int ipcu_search_IBlattice_##S(T *items, int IB_index, int *lattice_id, int *neib, T *posx, T *posy, T *posz,  \
                                T *posw, int64_t nthreads, ipcu_stream_t stream);                             \
  /* ibm.cu:68-85 SPM */                                                                                       \
  int ipcu_SPM_##S(T *items, T Radius, T *posB, T *f, T *ftmp, T *tau, T *posx, T *posy, T *Fx, T *Fy, T *Fz,   \
                   T *velx, T *vely, T *velz, T *velw, int64_t nthreads, ipcu_stream_t stream);               \
  /* ibm.cu:16-29 set_quaternionS (host: quaS is a host array) */                                              \
  void ipcu_set_quaternionS_##S(int IB_index, T q0, T q1, T q2, T q3, T *quaS);

IPCU_LEGACY_DECLS(float, f32)
IPCU_LEGACY_DECLS(double, f64)

/* ibm.cu:276-344 IB_directForcing (float only in the reference) */
int ipcu_IB_directForcing_f32(float *items, int *lattice_id, int *neib, float *posx, float *posy, float *posz,
                              float *posw, float *velx, float *vely, float *velz, float *velw, float *Fx,
                              float *Fy, float *Fz, float *Gw, int64_t nthreads, ipcu_stream_t stream);
/* ibm.cu:87-122 SPM_ellipse (float only in the reference) */
int ipcu_SPM_ellipse_f32(float *items, float Rada, float Radb, float *quaS, float *posB, float *f, float *tau,
                         float *posx, float *posy, float *posz, float *velx, float *vely, float *velz,
                         float *velB, float *angleVB, int64_t nthreads, ipcu_stream_t stream);

/* ---------------------------------------------------------------------
 * Host set-up helpers (all pointers are HOST pointers)
 * --------------------------------------------------------------------- */
/* basic.cu:70-98 Items::setc: c = dx/dt, tau, taus, and c-scaled
 * velocity components and weights (27 entries each, Q used). */
int ipcu_setc(int Q, double dx, double dt, int alpha, double *c, double *tau, double *taus, double *cx,
              double *cy, double *cz, double *w);
/* basic.cu:157-170 read_M: reads <dir>/input/{MRT,Minv,S}_D3Q<Q>.csv */
int ipcu_read_M_csv(const char *dir, int Q, double *M, double *S, double *Minv);
/* basic.cu:171-201 set_M: zeroes the shear rates in S and forms MM = Minv diag(S) M */
int ipcu_set_M(int Q, const double *M_in, const double *S_in, const double *Minv_in, double *M, double *S,
               double *Minv, double *MM);
/* basic.cu:203-237 set_neibghor_wall: appends one ghost per open fluid
 * cell to `neib` (room for `cap` cells); owner_out[g] = owner of ghost g.
 * Returns the ghost count (num_wall) or a negative status. */
int64_t ipcu_set_neibghor_wall(int Q, int nx, int ny, int nz, int64_t num_calc, const int *lnum, int *neib,
                               int64_t cap, int *owner_out);
/* set_bound.cu:23-38 set_walln: six wall lists (room for `cap` each) */
int ipcu_set_walln_f32(const float *items, const int *neib, int64_t cap, int *const *wall_out, int *sizes);
int ipcu_set_walln_f64(const double *items, const int *neib, int64_t cap, int *const *wall_out, int *sizes);
/* set_bound.cu:40-162 set_bound2D / set_bound3D: nextK, nextB (num_wall*Q) */
int ipcu_set_bound2D_f32(const float *items, int num_block, const int *neib, int *nextK, int *nextB);
int ipcu_set_bound2D_f64(const double *items, int num_block, const int *neib, int *nextK, int *nextB);
int ipcu_set_bound3D_f32(const float *items, int num_block, const int *neib, int *nextK, int *nextB);
int ipcu_set_bound3D_f64(const double *items, int num_block, const int *neib, int *nextK, int *nextB);
/* The case drivers' box numbering with divx/divy refinement
 * (LockExchange/LockExchange.cu:34-127). Returns num_calc. */
int64_t ipcu_build_box_grid(int Q, int nx0, int ny0, int nz, double dx, double ratiox, double ratioy,
                            const int *divx, const int *divy, int *lnum, int *neib, double *posx, double *posy,
                            double *posz, double *delX, double *delY);

/* ---------------------------------------------------------------------
 * Device geometry set-up (all array pointers are DEVICE pointers; divx and
 * divy are host arrays). Replaces the case drivers' host loops.
 * --------------------------------------------------------------------- */
/* LockExchange/LockExchange.cu:55-127 + basic.cu:203-237 on the GPU: box
 * numbering lnum[NX*NY*nz], neighbour table neib[cap*Q] with one ghost per
 * open cell (ghost numbering in the reference's scan order), cell geometry
 * pos*, del* (cap entries; ghosts copy their owner), owner[num_wall].
 * Returns IPCU_ERR_CAPACITY when num_calc + num_wall > cap. Synchronises
 * `stream`; allocates small temporaries. */
int ipcu_build_box_device_f32(int Q, int nx0, int ny0, int nz, double dx, double ratiox, double ratioy,
                              const int *divx, const int *divy, int *lnum, int *neib, float *posx, float *posy,
                              float *posz, float *delX, float *delY, int64_t cap, int *owner, int64_t *num_calc,
                              int64_t *num_wall, ipcu_stream_t stream);
int ipcu_build_box_device_f64(int Q, int nx0, int ny0, int nz, double dx, double ratiox, double ratioy,
                              const int *divx, const int *divy, int *lnum, int *neib, double *posx, double *posy,
                              double *posz, double *delX, double *delY, int64_t cap, int *owner,
                              int64_t *num_calc, int64_t *num_wall, ipcu_stream_t stream);
/* SphereFallSuzuki2018/SphereSuzuki.cu:268-275: lattice_id[m] = the fluid
 * cell (index < num_calc) nearest marker m (posw[3m..3m+2]); first index
 * among equal distances. Asynchronous on `stream`. */
int ipcu_nearest_cells_f32(const float *posx, const float *posy, const float *posz, int64_t num_calc,
                           const float *posw, int num_markers, int *lattice_id, ipcu_stream_t stream);
int ipcu_nearest_cells_f64(const double *posx, const double *posy, const double *posz, int64_t num_calc,
                           const double *posw, int num_markers, int *lattice_id, ipcu_stream_t stream);

/* pybind_LockExchange/kernel.cu:4-17 (the prototype's kernel): data[i] += value */
int ipcu_add_scalar_f32(float *data, int64_t n, float value, ipcu_stream_t stream);

/* ======================================================================
 * 2. Structured-grid solver (fused B200 path)
 * ====================================================================== */
#include "ipcu_sim.h"
#include "ipcu_sim3d.h"

#ifdef __cplusplus
}
#endif
#endif /* IPCU_H */
