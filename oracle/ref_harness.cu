// Test infrastructure only: a C-ABI harness around the UNMODIFIED reference
// kernel library (function/*.cu of Kasahara1341/IP_CU_LBM), compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/libipcu_ref.so.
//
// It exists so that tests and the reference arm of bench.py can run the
// reference's own CUDA code on the same device buffers as the product:
//   * ref_<kernel>_<f32|f64>  launch one reference kernel exactly as the case
//     drivers do (<<<ceil(n/64), 64>>> on the legacy default stream) and
//     synchronise (ref: LockExchange/LockExchange.cu:195-196);
//   * ref_* host wrappers call the reference's host set-up functions
//     (set_neibghor_wall, set_walln, set_bound2D/3D, set_M, Items::setc);
//   * ref_le_steps / ref_ibm_steps replay the case drivers' per-step kernel
//     order (ref: LockExchange/LockExchange.cu:214-278,
//     EllipticalFall2/EllipticalFallxz.cu:344-430).
// Nothing in the product links or loads this library.
#include "all.hpp"
#include <unistd.h>

// set_out is defined in function/adv.cu with (posx, posy) arguments that the
// declaration in all.hpp lacks; declare the defined form.
template <typename Typ>
__global__ void set_out(Typ *items, int *neib, Typ *ftmp, Typ *fout, Typ *fin, Typ *finy, Typ *posx,
                        Typ *posy, Typ *delX, Typ *delY);

namespace {
constexpr int kBS = 64;
inline int nblk(long long n) { return (int)((n + kBS - 1) / kBS); }
inline int fin_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  return (int)cudaDeviceSynchronize();
}
// driver-local copy kernel of EllipticalFall2/EllipticalFallxz.cu:4-13
template <typename Typ>
__global__ void h_set_f_ftmp(Typ *items, Typ *f, Typ *ftmp) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id < items[IDX_num_calc]) {
    int q = (int)items[IDX_Q];
    for (int k = 0; k < q; k++) ftmp[id * q + k] = f[id * q + k];
  }
}
}  // namespace

#define REF_BOTH(X) X(float, f32) X(double, f64)

// ---------------------------------------------------------------- collision.cu
#define DEF(T, S)                                                                                   \
  extern "C" int ref_equ_f_##S(T *it, T *feq, T *p, T *u, T *v, T *w, long long n) {                \
    equ_f<T><<<nblk(n), kBS>>>(it, feq, p, u, v, w);                                                \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_equ_g_##S(T *it, T *feq, T *s, T *u, T *v, T *w, long long n) {                \
    equ_g<T><<<nblk(n), kBS>>>(it, feq, s, u, v, w);                                                \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_wall_function_##S(T *it, T *dX, T *dY, int x, int y, int z, int nw, int *wall,  \
                                       T *u, T *v, T *w, T *Fx, T *Fy, T *rho, long long n) {        \
    wall_function<T><<<nblk(n), kBS>>>(it, dX, dY, x, y, z, nw, wall, u, v, w, Fx, Fy, rho);         \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_Force_##S(T *it, int bf, int *neib, T *f, T *feq, T *tau, T *Fk, T *Fx, T *Fy,  \
                               T *Fz, T *p, T *rho, T *sal, T *phi, T *u, T *v, T *w, T *dX, T *dY,  \
                               T *px, T *py, T *pz, long long n) {                                   \
    Force<T><<<nblk(n), kBS>>>(it, bf != 0, neib, f, feq, tau, Fk, Fx, Fy, Fz, p, rho, sal, phi, u,  \
                               v, w, dX, dY, px, py, pz);                                           \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_col_f_MRT_##S(T *it, T *tau, T *f, T *ftmp, T *feq, T *Fk, T *M, T *Minv, T *Sv, \
                                   T *MM, long long n) {                                            \
    col_f_MRT<T><<<nblk(n), kBS>>>(it, tau, f, ftmp, feq, Fk, M, Minv, Sv, MM);                      \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_col_f_SRT_##S(T *it, T *tau, T *f, T *ftmp, T *feq, T *Fk, long long n) {       \
    col_f_SRT<T><<<nblk(n), kBS>>>(it, tau, f, ftmp, feq, Fk);                                      \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_col_g_reg_##S(T *it, T *taus, T *g, T *gtmp, T *geq, T *s, T *u, T *v, T *w,   \
                                   long long n) {                                                   \
    col_g_reg<T><<<nblk(n), kBS>>>(it, taus, g, gtmp, geq, s, u, v, w);                              \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_col_PF_##S(T *it, int *neib, T *taus, T *g, T *gtmp, T *geq, T *phi, T *u, T *v, \
                                T *w, T *phio, T *uo, T *vo, T *wo, T *px, T *py, T *pz,            \
                                long long n) {                                                      \
    col_PF<T><<<nblk(n), kBS>>>(it, neib, taus, g, gtmp, geq, phi, u, v, w, phio, uo, vo, wo, px,    \
                                py, pz);                                                            \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_update_scalar_##S(T *it, T *g, T *s, long long n) {                            \
    update_scalar<T><<<nblk(n), kBS>>>(it, g, s);                                                   \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_update_rho_##S(T *it, T rhoL, T rhoH, T *f, T *Fx, T *Fy, T *Fz, T *p, T *sal,  \
                                    T *phi, T *rho, T *u, T *v, T *w, long long n) {                 \
    update_rho<T><<<nblk(n), kBS>>>(it, rhoL, rhoH, f, Fx, Fy, Fz, p, sal, phi, rho, u, v, w);       \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_resetF_##S(T *it, T *Fx, T *Fy, T *Fz, int num_F, long long n) {               \
    resetF<T><<<nblk(n), kBS>>>(it, Fx, Fy, Fz, num_F);                                             \
    return fin_launch();                                                                            \
  }
REF_BOTH(DEF)
#undef DEF

// ---------------------------------------------------------------- adv.cu, propagation.cu, set_bound.cu, basic.cu
#define DEF(T, S)                                                                                   \
  extern "C" int ref_set_wall_f_##S(T *it, int *neib, T *f, long long n) {                          \
    set_wall_f<T><<<nblk(n), kBS>>>(it, neib, f);                                                   \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_set_out_##S(T *it, int *neib, T *ftmp, T *fout, T *fin, T *finy, T *px, T *py,  \
                                 T *dX, T *dY, long long n) {                                        \
    set_out<T><<<nblk(n), kBS>>>(it, neib, ftmp, fout, fin, finy, px, py, dX, dY);                   \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_set_fin_##S(T *it, int *neib, int *nextK, T *fin, T *finy, long long n) {      \
    set_fin<T><<<nblk(n), kBS>>>(it, neib, nextK, fin, finy);                                       \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_reset_f_##S(T *it, T *ftmp, T *fin, T *f, long long n) {                       \
    reset_f<T><<<nblk(n), kBS>>>(it, ftmp, fin, f);                                                 \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_set_wall_f_inv_##S(T *it, int *neib, int *nextB, int *nextK, T *f,             \
                                        long long n) {                                              \
    set_wall_f_inv<T><<<nblk(n), kBS>>>(it, neib, nextB, nextK, f);                                 \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_set_tmp_##S(T *it, int *neib, T *f, T *ftmp, T *fout, T *fin, long long n) {    \
    set_tmp<T><<<nblk(n), kBS>>>(it, neib, f, ftmp, fout, fin);                                     \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_IP_process_##S(T *it, int *neib, T *f, T *feq, T *ftmp, T *fout, int *nextB,   \
                                    int *nextK, T *px, T *py, T *dX, T *dY, int slip, long long n) { \
    IP_process<T>(it, nblk(n), kBS, neib, f, feq, ftmp, fout, nextB, nextK, px, py, dX, dY, slip);   \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_set_wall_propagation_##S(T *it, int bc, int *neib, int *nextK, int *nextB,      \
                                              T *ftmp, long long n) {                               \
    set_wall_propagation<T><<<nblk(n), kBS>>>(it, bc, neib, nextK, nextB, ftmp);                    \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_propagation_##S(T *it, int *neib, T *f, T *ftmp, long long n) {                \
    propagation<T><<<nblk(n), kBS>>>(it, neib, f, ftmp);                                            \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_set_wall_rho_##S(T *it, int *neib, T *rho, long long n) {                      \
    set_wall_rho<T><<<nblk(n), kBS>>>(it, neib, rho);                                               \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_reset_pressure_##S(T *it, T *p, T *f, T *u, T *v, T *w, T alpha, long long n) { \
    reset_pressure<T><<<nblk(n), kBS>>>(it, p, f, u, v, w, alpha);                                   \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_reset_wall_fin_##S(T *it, T *fin, T *finy, long long n) {                      \
    reset_wall_fin<T><<<nblk(n), kBS>>>(it, fin, finy);                                             \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_LES_##S(T *it, int *neib, T *tau, T *taus, T *phi, T *rho, T muL, T muH, T *u,  \
                             T *v, T *w, T *px, T *py, T *pz, long long n) {                         \
    LES<T><<<nblk(n), kBS>>>(it, neib, tau, taus, phi, rho, muL, muH, u, v, w, px, py, pz);          \
    return fin_launch();                                                                            \
  }
REF_BOTH(DEF)
#undef DEF

// ---------------------------------------------------------------- ibm.cu
#define DEF(T, S)                                                                                   \
  extern "C" int ref_get_IBMGw2_##S(T *it, int *lid, int *neib, T *f, T *tau, T *px, T *py, T *pz,   \
                                    T *posw, T *posB, T *nB, T *u, T *v, T *w, T *velw, T *Fx,       \
                                    T *Fy, T *Fz, T *Gw, T rhof, long long n) {                      \
    get_IBMGw2<T><<<nblk(n), kBS>>>(it, lid, neib, f, tau, px, py, pz, posw, posB, nB, u, v, w,      \
                                    velw, Fx, Fy, Fz, Gw, rhof);                                    \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_update_velIBM_##S(T *it, int *lid, T *f, T *ftmp, T *p, T *tau, T *u, T *v,     \
                                       T *w, T *uo, T *vo, T *wo, T *Fx, T *Fy, T *Fz, long long n) {  \
    update_velIBM<T><<<nblk(n), kBS>>>(it, lid, f, ftmp, p, tau, u, v, w, uo, vo, wo, Fx, Fy, Fz);   \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_update_IBbody_##S(T *it, int ib, T *massB, T *densB, T *inertia, T *FB,         \
                                       T *posB, T *Torque, T *velB, T *quat, T *quaS, T *angleVB,    \
                                       T *posw, T *Gw, T *quatold, T rhof, long long n) {           \
    update_IBbody<T><<<nblk(n), kBS>>>(it, ib, massB, densB, inertia, FB, posB, Torque, velB, quat,  \
                                       quaS, angleVB, posw, Gw, quatold, rhof);                     \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_update_IBpoint_##S(T *it, int ib, T *posB, T *velB, T *angleVB, T *quaS,        \
                                        T *posw, T *oposw, T *nB, T *onB, T *velw, long long n) {    \
    update_IBpoint<T><<<nblk(n), kBS>>>(it, ib, posB, velB, angleVB, quaS, posw, oposw, nB, onB,     \
                                        velw);                                                      \
    return fin_launch();                                                                            \
  }                                                                                                 \
  extern "C" int ref_SPM_##S(T *it, T R, T *posB, T *f, T *ftmp, T *tau, T *px, T *py, T *Fx, T *Fy, \
                             T *Fz, T *u, T *v, T *w, T *velw, long long n) {                        \
    SPM<T><<<nblk(n), kBS>>>(it, R, posB, f, ftmp, tau, px, py, Fx, Fy, Fz, u, v, w, velw);          \
    return fin_launch();                                                                            \
  }
REF_BOTH(DEF)
#undef DEF

extern "C" int ref_search_IBlattice_f32(float *it, int ib, int *lid, int *neib, float *px, float *py,
                                        float *pz, float *posw, long long n) {
  search_IBlattice<float><<<nblk(n), kBS>>>(it, ib, lid, neib, px, py, pz, posw);
  return fin_launch();
}
extern "C" int ref_SPM_ellipse_f32(float *it, float a, float b, float *quaS, float *posB, float *f,
                                   float *tau, float *px, float *py, float *pz, float *u, float *v,
                                   float *w, float *velB, float *angleVB, long long n) {
  SPM_ellipse<float><<<nblk(n), kBS>>>(it, a, b, quaS, posB, f, tau, px, py, pz, u, v, w, velB,
                                       angleVB);
  return fin_launch();
}
extern "C" int ref_IB_directForcing_f32(float *it, int *lid, int *neib, float *px, float *py,
                                        float *pz, float *posw, float *u, float *v, float *w,
                                        float *velw, float *Fx, float *Fy, float *Fz, float *Gw,
                                        long long n) {
  IB_directForcing<<<nblk(n), kBS>>>(it, lid, neib, px, py, pz, posw, u, v, w, velw, Fx, Fy, Fz,
                                     Gw);
  return fin_launch();
}

// ---------------------------------------------------------------- host set-up wrappers
// Items::setc (ref: function/basic.cu:70-98). Outputs c, tau, taus and the
// per-direction tables (27 entries each).
extern "C" void ref_setc(int Q, double dx, double dt, int alpha, double *c, double *tau,
                         double *taus, double *cx, double *cy, double *cz, double *w) {
  Items it;
  it.num_velocity = Q;
  it.dx = dx;
  it.dt = dt;
  it.setc(alpha);
  *c = it.c;
  *tau = it.tau;
  *taus = it.taus;
  for (int k = 0; k < 27; k++) {
    cx[k] = it.cx[k];
    cy[k] = it.cy[k];
    cz[k] = it.cz[k];
    w[k] = (k < Q) ? it.weight[k] : 0.0;
  }
}

// set_M (ref: function/basic.cu:172-201) reads input/{MRT,S,Minv}_D3Q<Q>.csv
// relative to the working directory; `dir` is the directory holding input/.
extern "C" int ref_set_M_f64(const char *dir, int Q, double *M, double *S, double *Minv,
                             double *MM) {
  char old[4096];
  if (!getcwd(old, sizeof old)) return -1;
  if (chdir(dir) != 0) return -2;
  std::vector<double> vM(Q * Q), vS(Q), vMi(Q * Q), vMM(Q * Q);
  set_M<double>(Q, vM, vS, vMi, vMM);
  if (chdir(old) != 0) return -3;
  for (int i = 0; i < Q * Q; i++) {
    M[i] = vM[i];
    Minv[i] = vMi[i];
    MM[i] = vMM[i];
  }
  for (int i = 0; i < Q; i++) S[i] = vS[i];
  return 0;
}

// set_neibghor_wall (ref: function/basic.cu:204-237). Grows every per-cell
// array by one ghost per boundary cell. Per-cell inputs have num_calc
// entries (Q per cell for f, g, Fk); outputs have room for `cap` cells.
// Returns the new total cell count, or -1 if `cap` is too small.
extern "C" long long ref_set_neibghor_wall_f32(
    int nx, int ny, int nz, int Q, int num_calc, const int *lnum, const int *divx, const int *divy,
    const int *neib_in, const float *const *cell_in /*11: p,rho,phi,px,py,pz,dX,dY,u,v,w*/,
    const float *const *q_in /*3: f,g,Fk*/, long long cap, int *neib_out,
    float *const *cell_out, float *const *q_out) {
  Items it;
  it.nx = nx;
  it.ny = ny;
  it.nz = nz;
  it.num_velocity = Q;
  it.num_calc = num_calc;
  std::vector<int> vl(lnum, lnum + (long long)nx * ny * nz), vdx(divx, divx + nx),
      vdy(divy, divy + ny), vn(neib_in, neib_in + (long long)num_calc * Q);
  std::vector<float> c[11], q[3];
  for (int i = 0; i < 11; i++) c[i].assign(cell_in[i], cell_in[i] + num_calc);
  for (int i = 0; i < 3; i++) q[i].assign(q_in[i], q_in[i] + (long long)num_calc * Q);
  set_neibghor_wall<float>(it, vl, vdx, vdy, vn, q[0], q[1], q[2], c[0], c[1], c[2], c[3], c[4], c[5],
                           c[6], c[7], c[8], c[9], c[10]);
  long long nt = (long long)c[0].size();
  if (nt > cap) return -1;
  for (long long i = 0; i < nt * Q; i++) neib_out[i] = vn[i];
  for (int a = 0; a < 11; a++)
    for (long long i = 0; i < nt; i++) cell_out[a][i] = c[a][i];
  for (int a = 0; a < 3; a++)
    for (long long i = 0; i < nt * Q; i++) q_out[a][i] = q[a][i];
  return nt;
}

// set_walln (ref: function/set_bound.cu:23-38); wall lists written to
// wall_out[0..5] (room for `cap` each), sizes to sizes[6].
extern "C" int ref_set_walln_f32(const float *items, int nitems, const int *neib, long long nneib,
                                 long long cap, int *const *wall_out, int *sizes) {
  std::vector<float> it(items, items + nitems);
  std::vector<int> vn(neib, neib + nneib), w[6];
  set_walln<float>(it, vn, w[0], w[1], w[2], w[3], w[4], w[5]);
  for (int a = 0; a < 6; a++) {
    if ((long long)w[a].size() > cap) return -1;
    sizes[a] = (int)w[a].size();
    for (size_t i = 0; i < w[a].size(); i++) wall_out[a][i] = w[a][i];
  }
  return 0;
}

// set_bound2D / set_bound3D (ref: function/set_bound.cu:40-162). nextK/nextB
// get num_wall*Q entries.
extern "C" int ref_set_bound_f32(int dim, const float *items, int nitems, int num_block,
                                 const int *neib, long long nneib, int *nextK, int *nextB) {
  std::vector<float> it(items, items + nitems);
  std::vector<int> vn(neib, neib + nneib), vk, vb;
  if (dim == 2)
    set_bound2D<float>(it, num_block, vn, vk, vb);
  else
    set_bound3D<float>(it, num_block, vn, vk, vb);
  for (size_t i = 0; i < vk.size(); i++) {
    nextK[i] = vk[i];
    nextB[i] = vb[i];
  }
  return (int)vk.size();
}

extern "C" void ref_set_quaternionS_f32(float q0, float q1, float q2, float q3, float *quaS) {
  set_quaternionS<float>(0, q0, q1, q2, q3, quaS);
}

// ---------------------------------------------------------------- step chains
// Buffer slots for the step chains (device pointers).
enum RefBuf {
  B_items, B_neib, B_nextB, B_nextK, B_f, B_ftmp, B_fout, B_feq, B_Fk, B_g, B_p, B_sal, B_phi, B_tau,
  B_taus, B_Fx, B_Fy, B_Fz, B_rho, B_px, B_py, B_pz, B_dX, B_dY, B_u, B_v, B_w, B_M, B_Minv, B_S, B_MM,
  B_w1, B_w2, B_w3, B_w4, B_w5, B_w6,
  // IBM
  B_lid, B_uo, B_vo, B_wo, B_massB, B_densB, B_inertia, B_FB, B_posB, B_Torque, B_velB, B_quat,
  B_quaS, B_angleVB, B_posw, B_oposw, B_Gw, B_velw, B_nB, B_onB, B_quatold,
  B_COUNT
};

// LockExchange step order (ref: LockExchange/LockExchange.cu:214-278).
// ip[]: 0 n_threads, 1 nsteps, 2 slip(0)/bounce-back(1), 3 use_mrt, 4 use_scalar,
//       5 use_wall_function, 6 boussi, 7..12 wall sizes, 13 num_F
// fp[]: 0 rhoL, 1 rhoH
extern "C" int ref_le_steps_f32(void *const *b, const long long *ip, const float *fp) {
  long long n = ip[0];
  int nb = nblk(n);
  float *it = (float *)b[B_items];
  int *neib = (int *)b[B_neib];
#define F(x) ((float *)b[x])
#define I(x) ((int *)b[x])
  for (long long s = 0; s < ip[1]; s++) {
    if (ip[5]) {
      wall_function<float><<<nb, kBS>>>(it, F(B_dX), F(B_dY), 1, 0, 0, (int)ip[7], I(B_w1), F(B_v), F(B_w), F(B_u), F(B_Fy), F(B_Fz), F(B_rho));
      wall_function<float><<<nb, kBS>>>(it, F(B_dX), F(B_dY), 1, 0, 0, (int)ip[9], I(B_w3), F(B_v), F(B_w), F(B_u), F(B_Fy), F(B_Fz), F(B_rho));
      wall_function<float><<<nb, kBS>>>(it, F(B_dX), F(B_dY), 0, 0, 1, (int)ip[11], I(B_w5), F(B_u), F(B_v), F(B_w), F(B_Fx), F(B_Fy), F(B_rho));
      wall_function<float><<<nb, kBS>>>(it, F(B_dX), F(B_dY), 0, 0, 1, (int)ip[12], I(B_w6), F(B_u), F(B_v), F(B_w), F(B_Fx), F(B_Fy), F(B_rho));
      wall_function<float><<<nb, kBS>>>(it, F(B_dX), F(B_dY), 0, 1, 0, (int)ip[8], I(B_w2), F(B_u), F(B_w), F(B_v), F(B_Fx), F(B_Fz), F(B_rho));
      wall_function<float><<<nb, kBS>>>(it, F(B_dX), F(B_dY), 0, 1, 0, (int)ip[10], I(B_w4), F(B_u), F(B_w), F(B_v), F(B_Fx), F(B_Fz), F(B_rho));
    }
    equ_f<float><<<nb, kBS>>>(it, F(B_feq), F(B_p), F(B_u), F(B_v), F(B_w));
    Force<float><<<nb, kBS>>>(it, ip[6] != 0, neib, F(B_f), F(B_feq), F(B_tau), F(B_Fk), F(B_Fx), F(B_Fy), F(B_Fz), F(B_p), F(B_rho), F(B_sal), F(B_phi), F(B_u), F(B_v), F(B_w), F(B_dX), F(B_dY), F(B_px), F(B_py), F(B_pz));
    if (ip[3])
      col_f_MRT<float><<<nb, kBS>>>(it, F(B_tau), F(B_f), F(B_ftmp), F(B_feq), F(B_Fk), F(B_M), F(B_Minv), F(B_S), F(B_MM));
    else
      col_f_SRT<float><<<nb, kBS>>>(it, F(B_tau), F(B_f), F(B_ftmp), F(B_feq), F(B_Fk));
    IP_process<float>(it, nb, kBS, neib, F(B_f), F(B_feq), F(B_ftmp), F(B_fout), I(B_nextB), I(B_nextK), F(B_px), F(B_py), F(B_dX), F(B_dY), (int)ip[2]);
    if (ip[4]) {
      col_g_reg<float><<<nb, kBS>>>(it, F(B_taus), F(B_g), F(B_ftmp), F(B_feq), F(B_sal), F(B_u), F(B_v), F(B_w));
      IP_process<float>(it, nb, kBS, neib, F(B_g), F(B_feq), F(B_ftmp), F(B_fout), I(B_nextB), I(B_nextK), F(B_px), F(B_py), F(B_dX), F(B_dY), (int)ip[2]);
      update_scalar<float><<<nb, kBS>>>(it, F(B_g), F(B_sal));
    }
    update_rho<float><<<nb, kBS>>>(it, fp[0], fp[1], F(B_f), F(B_Fx), F(B_Fy), F(B_Fz), F(B_p), F(B_sal), F(B_phi), F(B_rho), F(B_u), F(B_v), F(B_w));
    set_wall_rho<float><<<nb, kBS>>>(it, neib, F(B_rho));
    resetF<float><<<nb, kBS>>>(it, F(B_Fx), F(B_Fy), F(B_Fz), (int)ip[13]);
  }
  return fin_launch();
}

// Moving-IBM step order (ref: EllipticalFall2/EllipticalFallxz.cu:344-430;
// SphereFallSuzuki2018/SphereSuzuki.cu:369-455).
// ip[]: 0 n_threads, 1 nsteps, 2 bc, 3 use_mrt, 6 boussi, 13 num_F, 14 num_Gw
// fp[]: 0 rhoL, 1 rhoH
extern "C" int ref_ibm_steps_f32(void *const *b, const long long *ip, const float *fp) {
  long long n = ip[0];
  int nb = nblk(n);
  float *it = (float *)b[B_items];
  int *neib = (int *)b[B_neib];
  for (long long s = 0; s < ip[1]; s++) {
    equ_f<float><<<nb, kBS>>>(it, F(B_feq), F(B_p), F(B_u), F(B_v), F(B_w));
    Force<float><<<nb, kBS>>>(it, ip[6] != 0, neib, F(B_f), F(B_feq), F(B_tau), F(B_Fk), F(B_Fx), F(B_Fy), F(B_Fz), F(B_p), F(B_rho), F(B_sal), F(B_phi), F(B_u), F(B_v), F(B_w), F(B_dX), F(B_dY), F(B_px), F(B_py), F(B_pz));
    if (ip[3])
      col_f_MRT<float><<<nb, kBS>>>(it, F(B_tau), F(B_f), F(B_ftmp), F(B_feq), F(B_Fk), F(B_M), F(B_Minv), F(B_S), F(B_MM));
    else
      col_f_SRT<float><<<nb, kBS>>>(it, F(B_tau), F(B_f), F(B_ftmp), F(B_feq), F(B_Fk));
    IP_process<float>(it, nb, kBS, neib, F(B_f), F(B_feq), F(B_ftmp), F(B_fout), I(B_nextB), I(B_nextK), F(B_px), F(B_py), F(B_dX), F(B_dY), (int)ip[2]);
    update_rho<float><<<nb, kBS>>>(it, fp[0], fp[1], F(B_f), F(B_Fx), F(B_Fy), F(B_Fz), F(B_p), F(B_sal), F(B_phi), F(B_rho), F(B_u), F(B_v), F(B_w));
    resetF<float><<<nb, kBS>>>(it, F(B_Fx), F(B_Fy), F(B_Fz), (int)ip[13]);
    h_set_f_ftmp<float><<<nb, kBS>>>(it, F(B_f), F(B_ftmp));
    get_IBMGw2<float><<<nb, kBS>>>(it, I(B_lid), neib, F(B_f), F(B_tau), F(B_px), F(B_py), F(B_pz), F(B_posw), F(B_posB), F(B_nB), F(B_u), F(B_v), F(B_w), F(B_velw), F(B_Fx), F(B_Fy), F(B_Fz), F(B_Gw), fp[1]);
    update_velIBM<float><<<nb, kBS>>>(it, I(B_lid), F(B_f), F(B_ftmp), F(B_p), F(B_tau), F(B_u), F(B_v), F(B_w), F(B_uo), F(B_vo), F(B_wo), F(B_Fx), F(B_Fy), F(B_Fz));
    update_IBbody<float><<<nb, kBS>>>(it, 0, F(B_massB), F(B_densB), F(B_inertia), F(B_FB), F(B_posB), F(B_Torque), F(B_velB), F(B_quat), F(B_quaS), F(B_angleVB), F(B_posw), F(B_Gw), F(B_quatold), fp[1]);
    update_IBpoint<float><<<nb, kBS>>>(it, 0, F(B_posB), F(B_velB), F(B_angleVB), F(B_quaS), F(B_posw), F(B_oposw), F(B_nB), F(B_onB), F(B_velw));
    search_IBlattice<float><<<nb, kBS>>>(it, 0, I(B_lid), neib, F(B_px), F(B_py), F(B_pz), F(B_posw));
    resetF<float><<<nb, kBS>>>(it, F(B_Fx), F(B_Fy), F(B_Fz), (int)ip[13]);
    resetF<float><<<nb, kBS>>>(it, F(B_Gw), F(B_Gw), F(B_Gw), (int)ip[14]);
  }
  return fin_launch();
#undef F
#undef I
}

extern "C" int ref_buf_count() { return B_COUNT; }
