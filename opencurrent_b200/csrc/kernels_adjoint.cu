// Hand-written adjoints of the advection stencils on a periodic MAC grid.
//
// Forward (kernels_flow.cu, after sol_selfadvection3ddev.cu:135-337 and
// sol_passiveadvection3ddev.cu:31-78), written as face fluxes:
//   passive:  dphi(p) = -sum_d ih_d (F_d(p + e_d) - F_d(p)),  F_d(f) = V_d[f] * sel(V_d[f], phi[f-e_d], phi[f])
//   self:     dq(p)   = -sum_d ih_d (G_qd(p) - G_qd(p - e_d)),
//             G_qd(c) = a_qd(c) * sel(a_qd(c), q[c], q[c+e_d]),  a_qd(c) = (V_d[c+e_d] + V_d[c+e_d-e_q]) / 2
// where sel is the first-order upwind choice (a < 0 ? right : left) or the centred mean.  The
// upwind choice is piecewise constant, so the Jacobian is that of the bilinear flux with the
// choice frozen.  The transposed Jacobian applied to an output cotangent L (scaled by the time
// step c) is evaluated as a gather: every cell collects the contributions of the fluxes that
// read it, so there are no atomics and the result is deterministic.  lambda_G = c * ih_d *
// (L[c + e_d] - L[c]) is the cotangent of one flux.  Indices wrap periodically (the forward
// reads the periodic ghost copies, which are the wrapped interior values).
#include "ocu_internal.h"

namespace ocub {

struct Wrap {
  long long xs, ys;
  int nx, ny, nz;
  __device__ __forceinline__ long long at(int i, int j, int k) const {
    i = i < 0 ? i + nx : (i >= nx ? i - nx : i);
    j = j < 0 ? j + ny : (j >= ny ? j - ny : j);
    k = k < 0 ? k + nz : (k >= nz ? k - nz : k);
    return (long long)i * xs + (long long)j * ys + k;
  }
};

template <int A, int D> struct Unit { static constexpr int v = A == D ? 1 : 0; };

template <typename T, int IT>
__device__ __forceinline__ T pick(T a, T x0, T x1) {
  if (IT == OCU_IT_FIRST_ORDER_UPWIND) return a < 0 ? x1 : x0;
  return (T)0.5 * (x1 + x0);
}
// d sel / d x0 and d sel / d x1 (for the frozen upwind choice)
template <typename T, int IT>
__device__ __forceinline__ T dpick0(T a) {
  if (IT == OCU_IT_FIRST_ORDER_UPWIND) return a < 0 ? (T)0 : (T)1;
  return (T)0.5;
}
template <typename T, int IT>
__device__ __forceinline__ T dpick1(T a) {
  if (IT == OCU_IT_FIRST_ORDER_UPWIND) return a < 0 ? (T)1 : (T)0;
  return (T)0.5;
}

// ---- passive advection ------------------------------------------------------------------------
// lam_phi_out[p] = L[p] + c * (d dphi/d phi)^T L ;  lam_V[p] += c * (d dphi/d V)^T L
template <typename T, int IT>
__global__ void __launch_bounds__(256) k_adj_passive(const T *__restrict__ u, const T *__restrict__ v,
                                                     const T *__restrict__ w, const T *__restrict__ phi,
                                                     const T *__restrict__ L, T *__restrict__ lam_phi,
                                                     T *__restrict__ lu, T *__restrict__ lv, T *__restrict__ lw, T c,
                                                     T ihx, T ihy, T ihz, Wrap g) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= g.nz || j >= g.ny || i >= g.nx) return;
  const long long p = g.at(i, j, k);
  const T lp = L[p];
  T acc = lp;
  // x faces p (between p-ex and p) and p+ex (between p and p+ex)
  {
    const long long m = g.at(i - 1, j, k), q = g.at(i + 1, j, k);
    const T lf0 = c * ihx * (lp - L[m]), lf1 = c * ihx * (L[q] - lp);
    const T a0 = u[p], a1 = u[q];
    lu[p] += lf0 * pick<T, IT>(a0, phi[m], phi[p]);
    acc += lf0 * a0 * dpick1<T, IT>(a0) + lf1 * a1 * dpick0<T, IT>(a1);
  }
  {
    const long long m = g.at(i, j - 1, k), q = g.at(i, j + 1, k);
    const T lf0 = c * ihy * (lp - L[m]), lf1 = c * ihy * (L[q] - lp);
    const T a0 = v[p], a1 = v[q];
    lv[p] += lf0 * pick<T, IT>(a0, phi[m], phi[p]);
    acc += lf0 * a0 * dpick1<T, IT>(a0) + lf1 * a1 * dpick0<T, IT>(a1);
  }
  {
    const long long m = g.at(i, j, k - 1), q = g.at(i, j, k + 1);
    const T lf0 = c * ihz * (lp - L[m]), lf1 = c * ihz * (L[q] - lp);
    const T a0 = w[p], a1 = w[q];
    lw[p] += lf0 * pick<T, IT>(a0, phi[m], phi[p]);
    acc += lf0 * a0 * dpick1<T, IT>(a0) + lf1 * a1 * dpick0<T, IT>(a1);
  }
  lam_phi[p] = acc;
}

// ---- self advection ---------------------------------------------------------------------------
template <typename T>
struct SelfFields {
  const T *V[3];  // u, v, w at the step's start
  const T *L[3];  // cotangents of du, dv, dw (already projected)
  T ih[3];
  T c;
};

// Flux G_qd at cell (i,j,k): its cotangent lg, advecting velocity a and transported value s.
template <typename T, int IT, int Q, int D>
__device__ __forceinline__ void flux_qd(const SelfFields<T> &f, const Wrap &g, int i, int j, int k, T &lg, T &a,
                                        T &s) {
  constexpr int dx = Unit<0, D>::v, dy = Unit<1, D>::v, dz = Unit<2, D>::v;
  constexpr int qx = Unit<0, Q>::v, qy = Unit<1, Q>::v, qz = Unit<2, Q>::v;
  const long long c0 = g.at(i, j, k), cd = g.at(i + dx, j + dy, k + dz);
  const long long cdq = g.at(i + dx - qx, j + dy - qy, k + dz - qz);
  a = (T)0.5 * (f.V[D][cd] + f.V[D][cdq]);
  s = pick<T, IT>(a, f.V[Q][c0], f.V[Q][cd]);
  lg = f.c * f.ih[D] * (f.L[Q][cd] - f.L[Q][c0]);
}

// Contributions to field F (0 u, 1 v, 2 w) at cell (i,j,k).
template <typename T, int IT, int F>
__device__ __forceinline__ T self_adj_field(const SelfFields<T> &f, const Wrap &g, int i, int j, int k) {
  T acc = 0, lg, a, s;
  constexpr int fx = Unit<0, F>::v, fy = Unit<1, F>::v, fz = Unit<2, F>::v;
  // (A) F advects every component q along its own direction D = F: fluxes G_qF(c) with
  //     c + e_F = p or c + e_F - e_q = p; each takes half of the flux cotangent times s
#define SELF_ADJ_A(QQ)                                                                                \
  {                                                                                                   \
    constexpr int qx = Unit<0, QQ>::v, qy = Unit<1, QQ>::v, qz = Unit<2, QQ>::v;                     \
    flux_qd<T, IT, QQ, F>(f, g, i - fx, j - fy, k - fz, lg, a, s);                                    \
    acc += lg * (T)0.5 * s;                                                                           \
    flux_qd<T, IT, QQ, F>(f, g, i - fx + qx, j - fy + qy, k - fz + qz, lg, a, s);                     \
    acc += lg * (T)0.5 * s;                                                                           \
  }
  SELF_ADJ_A(0)
  SELF_ADJ_A(1)
  SELF_ADJ_A(2)
#undef SELF_ADJ_A
  // (B) F is the transported value of G_Fd(p) (left value) and G_Fd(p - e_d) (right value)
#define SELF_ADJ_B(DD)                                                                                \
  {                                                                                                   \
    constexpr int ex = Unit<0, DD>::v, ey = Unit<1, DD>::v, ez = Unit<2, DD>::v;                     \
    flux_qd<T, IT, F, DD>(f, g, i, j, k, lg, a, s);                                                   \
    acc += lg * a * dpick0<T, IT>(a);                                                                 \
    flux_qd<T, IT, F, DD>(f, g, i - ex, j - ey, k - ez, lg, a, s);                                    \
    acc += lg * a * dpick1<T, IT>(a);                                                                 \
  }
  SELF_ADJ_B(0)
  SELF_ADJ_B(1)
  SELF_ADJ_B(2)
#undef SELF_ADJ_B
  return acc;
}

// lam_V[p] += c * (d dV/dt / d V)^T L  for V = u, v, w
template <typename T, int IT>
__global__ void __launch_bounds__(256) k_adj_self(SelfFields<T> f, T *__restrict__ lu, T *__restrict__ lv,
                                                  T *__restrict__ lw, Wrap g) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= g.nz || j >= g.ny || i >= g.nx) return;
  const long long p = g.at(i, j, k);
  lu[p] += self_adj_field<T, IT, 0>(f, g, i, j, k);
  lv[p] += self_adj_field<T, IT, 1>(f, g, i, j, k);
  lw[p] += self_adj_field<T, IT, 2>(f, g, i, j, k);
}

static inline Wrap make_wrap(const ocu_layout &L) { return Wrap{L.xstride, L.ystride, L.nx, L.ny, L.nz}; }

static inline void adj_shape(const ocu_layout &L, dim3 *grid, dim3 *block) {
  *block = dim3(32, 8);
  *grid = dim3((L.nz + 31) / 32, (L.ny + 7) / 8, L.nx);
}

template <typename T>
ocu_status launch_adj_passive(const T *u, const T *v, const T *w, const T *phi, const T *L, T *lam_phi, T *lu, T *lv,
                              T *lw, const ocu_layout &Lc, double c, double hx, double hy, double hz, int interp,
                              cudaStream_t s) {
  dim3 grid, block;
  adj_shape(Lc, &grid, &block);
  const Wrap g = make_wrap(Lc);
  if (interp == OCU_IT_FIRST_ORDER_UPWIND)
    k_adj_passive<T, OCU_IT_FIRST_ORDER_UPWIND><<<grid, block, 0, s>>>(u, v, w, phi, L, lam_phi, lu, lv, lw, (T)c,
                                                                      (T)(1 / hx), (T)(1 / hy), (T)(1 / hz), g);
  else if (interp == OCU_IT_SECOND_ORDER_CENTERED)
    k_adj_passive<T, OCU_IT_SECOND_ORDER_CENTERED><<<grid, block, 0, s>>>(u, v, w, phi, L, lam_phi, lu, lv, lw, (T)c,
                                                                         (T)(1 / hx), (T)(1 / hy), (T)(1 / hz), g);
  else
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] passive advection adjoint - invalid interpolation type %d", interp);
  return check_launch("k_adj_passive");
}

template <typename T>
ocu_status launch_adj_self(const T *u, const T *v, const T *w, const T *Lu, const T *Lv, const T *Lw, T *lu, T *lv,
                           T *lw, const ocu_layout &Lc, double c, double hx, double hy, double hz, int interp,
                           cudaStream_t s) {
  dim3 grid, block;
  adj_shape(Lc, &grid, &block);
  SelfFields<T> f;
  f.V[0] = u; f.V[1] = v; f.V[2] = w;
  f.L[0] = Lu; f.L[1] = Lv; f.L[2] = Lw;
  f.ih[0] = (T)(1 / hx); f.ih[1] = (T)(1 / hy); f.ih[2] = (T)(1 / hz);
  f.c = (T)c;
  const Wrap g = make_wrap(Lc);
  if (interp == OCU_IT_FIRST_ORDER_UPWIND)
    k_adj_self<T, OCU_IT_FIRST_ORDER_UPWIND><<<grid, block, 0, s>>>(f, lu, lv, lw, g);
  else if (interp == OCU_IT_SECOND_ORDER_CENTERED)
    k_adj_self<T, OCU_IT_SECOND_ORDER_CENTERED><<<grid, block, 0, s>>>(f, lu, lv, lw, g);
  else
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] self advection adjoint - invalid interpolation type %d", interp);
  return check_launch("k_adj_self");
}

#define INST(T)                                                                                              \
  template ocu_status launch_adj_passive<T>(const T *, const T *, const T *, const T *, const T *, T *, T *, T *, \
                                            T *, const ocu_layout &, double, double, double, double, int,        \
                                            cudaStream_t);                                                       \
  template ocu_status launch_adj_self<T>(const T *, const T *, const T *, const T *, const T *, const T *, T *,   \
                                         T *, T *, const ocu_layout &, double, double, double, double, int,       \
                                         cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace ocub
