// Two-colour SOR sweep in one pass over HBM, fed by TMA.
//
// A red-black sweep done as two in-place colour launches moves every array twice (each launch
// reads u and b and writes u: ~6N values per sweep).  Here a CTA owns a (j,k) tile of TJ x TK
// cells and marches along i over a run of planes; each plane of u_in and b (with a two-cell
// halo in j and a 16-byte halo in k) is brought into shared memory once by a 3-D TMA box load
// (cp.async.bulk.tensor + mbarrier), D planes ahead of use.  At step s the CTA
//   1. updates the first colour on plane s+1 over the tile plus a one-cell ring (these need only
//      old second-colour values: planes s..s+2 are resident),
//   2. updates the second colour on plane s (its neighbours on planes s-1, s, s+1 now hold
//      first-colour values),
//   3. writes plane s (both colours) to u_out with 16-byte stores, plus the ghost cells whose
//      source is on plane s (same rules as the colour kernels' fused ghost writes).
// So a sweep reads u and b once and writes u once (~3N), out of place (u_in -> u_out: CTAs read
// their neighbours' halos, so in-place writes would race).  Each cell is updated with the same
// relax arithmetic and the same neighbour values as the two colour launches, so the result is
// bit-identical to them.
//
// Work split: the (tile, plane) steps of the whole level are cut into equal contiguous ranges,
// one per resident CTA (tile-major, so a range is one or two runs of planes), so every SM gets
// the same number of steps in a single wave.
//
// Preconditions checked by the host (otherwise the caller uses the colour launches): every face
// is Dirichlet or Neumann and nz is a multiple of 8.  With such faces a ghost is read only by
// its own source cell, before that cell changes, so the ghosts of u_in are read exactly as the
// colour launches read them (from memory, whatever they hold).  Periodic faces are excluded:
// there a ghost's source lies on the opposite face and changes during the first colour.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "ghost_emit.cuh"
#include "mg_fused.h"
#include "ocu_internal.h"
#include "relax_math.cuh"
#include "tma_ptx.cuh"

namespace ocub {

template <typename T>
struct SweepTile {
  static constexpr int TJ = 16;                        // tile rows (j)
  static constexpr int TK = sizeof(T) == 4 ? 64 : 32;  // tile columns (k)
  static constexpr int H = 16 / (int)sizeof(T);        // k halo = one 16-byte TMA granule (>= 2)
  static constexpr int W = TK + 2 * H;                 // shared row pitch, elements
  static constexpr int R = TJ + 4;                     // rows j0-2 .. j0+TJ+1
  static constexpr int PLANE = W * R;                  // elements per plane buffer
  static constexpr int D = 2;                          // loads in flight beyond the live planes
  static constexpr int NU = 4 + D;                     // u plane buffers (s-1 .. s+2, + D)
  static constexpr int NB = 2 + D;                     // b plane buffers (s, s+1, + D)
  static constexpr int THREADS = 256;
  // plane buffers, then NU mbarriers, the abort word (8 bytes) and the barrier of the
  // timeout test (8 bytes); +128 to align the base by hand
  static constexpr size_t SMEM = (size_t)(NU + NB) * PLANE * sizeof(T) + NU * sizeof(unsigned long long) + 16 + 128;
  static_assert((PLANE * sizeof(T)) % 128 == 0, "TMA destinations stay 128-byte aligned");
};

struct SweepArgs {
  int nx, ny, nz;
  int gx, gy;
  int first_color;    // colour updated first (0 = red)
  int ntk;            // tiles along k
  long long steps;    // tiles * nx (plane steps of the whole level)
  int wait_limit;     // polls of a load wait before the launch gives up (kWaitLimit by default)
  int stall_test;     // testing the timeout path: first wait on a barrier nothing completes
};

// One relax update from shared memory at offset o of the current plane buffer.  `inner`: the
// cell is known to touch no face, so its diagonal is c.ld (the face terms would add nothing).
template <typename T>
__device__ __forceinline__ T sweep_update(const T *uc, const T *um, const T *up, const T *bp, int o, int i, int j,
                                          int k, bool inner, const SweepArgs &a, const RelaxCoefD<T> &c,
                                          const T *__restrict__ diag) {
  using S = SweepTile<T>;
  const T self = uc[o];
  const T res = relax_res<T>(self, bp[o], uc[o - 1], uc[o + 1], uc[o - S::W], uc[o + S::W], um[o], up[o], c);
  const T dg = inner ? c.ld : relax_dg<T>(i, j, k, a.nx, a.ny, a.nz, c, diag);
  return self + c.omega * res / dg;
}

template <typename T>
__global__ void __launch_bounds__(SweepTile<T>::THREADS, 3) k_relax_sweep2(
    const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_b, T *__restrict__ u_out,
    long long xs, long long ys, SweepArgs a, RelaxCoefD<T> c, const T *__restrict__ diag, GhostEmit<T> ge,
    int *__restrict__ err) {
  pdl_entry();
  using S = SweepTile<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations must be 128-byte aligned: align the base explicitly
  T *us = reinterpret_cast<T *>(smem_raw + ((128 - (smem_addr(smem_raw) & 127)) & 127));
  T *bs = us + S::NU * S::PLANE;
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(bs + S::NB * S::PLANE);
  int &abort_flag = *reinterpret_cast<int *>(bar + S::NU);
  unsigned long long *stall_bar = bar + S::NU + 1;  // never arrived at: only the timeout test waits on it

  const int cA = a.first_color, cB = !a.first_color;
  const unsigned bytes = (unsigned)(S::PLANE * sizeof(T));
  const long long lo = a.steps * blockIdx.x / gridDim.x, hi = a.steps * (blockIdx.x + 1) / gridDim.x;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int q = 0; q < S::NU; q++) mbar_init(&bar[q], 1);
    mbar_init(stall_bar, 1);
    mbar_init_fence();
    tma_prefetch_map(&tm_u);
    tma_prefetch_map(&tm_b);
  }
  __syncthreads();
  if (a.stall_test) {
    // the timeout path without a fault: a wait that nothing completes runs out of polls before
    // any load is issued, so the CTA has nothing in flight when it returns
    if (threadIdx.x == 0 && !mbar_wait_bounded(stall_bar, 0u, a.wait_limit)) {
      atomicOr(err, 1);
      abort_flag = 1;
    }
    __syncthreads();
    if (abort_flag) return;
  }

  int gbase = 0;   // loads are numbered across this CTA's runs: slot = g % NU (u), g % NB (b)
  int issued = 0;  // (thread 0) loads issued in the current run
  for (long long idx = lo; idx < hi;) {
    const int tile = (int)(idx / a.nx);
    const int ia = (int)(idx % a.nx);
    const int ib = (int)((long long)ia + (hi - idx) < a.nx ? ia + (hi - idx) : a.nx);
    idx += ib - ia;
    const int k0 = (tile % a.ntk) * S::TK, j0 = (tile / a.ntk) * S::TJ;
    const int nload = ib - ia + 4;  // u planes ia-2 .. ib+1 (b planes ia-1 .. ib ride along)
    // ring-1 region of the tile away from every y/z face
    const bool tile_inner = j0 - 1 >= 1 && j0 + S::TJ <= a.ny - 2 && k0 - 1 >= 1 && k0 + S::TK <= a.nz - 2;
    // u plane p is read when it is within one plane of an interior plane (ghost planes -1 and
    // nx included); b plane p only for interior planes.  Loads of other planes are skipped.
    auto issue = [&](int m) {  // load m of this run: u plane ia-2+m and, for m >= 2, b plane ia-3+m
      const int g = gbase + m;
      unsigned long long *bm = &bar[g % S::NU];
      const int pu = ia - 2 + m, pb = ia - 3 + m;
      const bool lu = pu >= -1 && pu <= a.nx, lb = m >= 2 && pb >= 0 && pb < a.nx;
      mbar_expect_tx(bm, (lu ? bytes : 0u) + (lb ? bytes : 0u));  // with 0 bytes: a plain arrive
      // view x = k + H: the box starts at k = k0 - H
      if (lu) tma_load_3d(us + (g % S::NU) * S::PLANE, &tm_u, k0, j0 - 2 + a.gy, pu + a.gx, bm);
      if (lb) tma_load_3d(bs + (g % S::NB) * S::PLANE, &tm_b, k0, j0 - 2 + a.gy, pb + a.gx, bm);
    };
    // buffers of the previous run may still be read (its last output): finish with them first
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0)
      for (issued = 0; issued < nload && issued < S::D + 3; issued++) issue(issued);

    const int nsteps = ib - ia + 2;  // s = ia-2 .. ib-1
    for (int n = 0; n < nsteps; n++) {
      const int s = ia - 2 + n;
      if (threadIdx.x == 0) {
        // loads 0..n+2 must have landed (step 0 also needs loads 0 and 1)
        for (int m = (n == 0 ? 0 : n + 2); m <= n + 2; m++) {
          const int g = gbase + m;
          if (!mbar_wait_bounded(&bar[g % S::NU], (unsigned)((g / S::NU) & 1), a.wait_limit)) {
            atomicOr(err, 1);
            abort_flag = 1;
            // let the copies already issued -- the one waited for included -- land before the
            // CTA's shared memory goes away (each wait again bounded, by the default limit)
            for (int q = m; q < issued; q++)
              mbar_wait_bounded(&bar[(gbase + q) % S::NU], (unsigned)(((gbase + q) / S::NU) & 1), kWaitLimit);
            break;
          }
        }
      }
      __syncthreads();
      if (abort_flag) return;
      const int g = gbase + n;

      // 1. first colour on plane s+1, tile + one-cell ring (interior cells only)
      const int pr = s + 1;
      if (pr >= 0 && pr < a.nx) {
        const bool inner = tile_inner && pr >= 1 && pr <= a.nx - 2;
        T *uc = us + ((g + 1) % S::NU) * S::PLANE;
        const T *um = us + (g % S::NU) * S::PLANE, *up = us + ((g + 2) % S::NU) * S::PLANE;
        const T *bp = bs + ((g + 2) % S::NB) * S::PLANE;
        constexpr int PAIRS = S::TK / 2 + 1;
        for (int q = threadIdx.x; q < (S::TJ + 2) * PAIRS; q += S::THREADS) {
          const int jr = q / PAIRS, t = q % PAIRS;
          const int j = j0 - 1 + jr;
          const int k = k0 - 1 + 2 * t + ((pr + j + cA + k0 + 1) & 1);
          if (j < 0 || j >= a.ny || k < 0 || k >= a.nz) continue;
          const int o = (jr + 1) * S::W + (k - k0 + S::H);
          uc[o] = sweep_update<T>(uc, um, up, bp, o, pr, j, k, inner, a, c, diag);
        }
      }
      __syncthreads();

      // 2. second colour on plane s (tile only)
      if (s >= ia) {
        const bool inner = tile_inner && s >= 1 && s <= a.nx - 2;
        T *uc = us + (g % S::NU) * S::PLANE;
        const T *um = us + ((g - 1) % S::NU) * S::PLANE, *up = us + ((g + 1) % S::NU) * S::PLANE;
        const T *bp = bs + ((g + 1) % S::NB) * S::PLANE;
        constexpr int HALF = S::TK / 2;
        for (int q = threadIdx.x; q < S::TJ * HALF; q += S::THREADS) {
          const int jr = q / HALF, t = q % HALF;
          const int j = j0 + jr;
          const int k = k0 + 2 * t + ((s + j + cB + k0) & 1);
          if (j >= a.ny || k >= a.nz) continue;
          const int o = (jr + 2) * S::W + (k - k0 + S::H);
          uc[o] = sweep_update<T>(uc, um, up, bp, o, s, j, k, inner, a, c, diag);
        }
      }
      // the next TMA overwrites buffers this CTA has written through the generic proxy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (threadIdx.x == 0 && issued < nload) issue(issued++);  // reuses the buffers of plane s-1

      // 3. plane s out, with the ghosts it is the source of
      if (s >= ia) {
        const T *uc = us + (g % S::NU) * S::PLANE;
        constexpr int V = 16 / (int)sizeof(T);
        constexpr int VPR = S::TK / V;
        T *dst_plane = u_out + (long long)s * xs;
        for (int q = threadIdx.x; q < S::TJ * VPR; q += S::THREADS) {
          const int jr = q / VPR, kv = (q % VPR) * V;
          const int j = j0 + jr, k = k0 + kv;
          if (j >= a.ny || k >= a.nz) continue;
          const uint4 v = *reinterpret_cast<const uint4 *>(uc + (jr + 2) * S::W + S::H + kv);
          *reinterpret_cast<uint4 *>(dst_plane + (long long)j * ys + k) = v;
        }
        if (s == 0 || s == a.nx - 1) {  // a face plane: every cell is a ghost source
          for (int q = threadIdx.x; q < S::TJ * S::TK; q += S::THREADS) {
            const int jr = q / S::TK, kk = q % S::TK;
            const int j = j0 + jr, k = k0 + kk;
            if (j >= a.ny || k >= a.nz) continue;
            ge.emit(s, j, k, uc[(jr + 2) * S::W + S::H + kk]);
          }
        } else if (j0 == 0 || j0 + S::TJ >= a.ny || k0 == 0 || k0 + S::TK >= a.nz) {
          // rows j = 0, ny-1 and columns k = 0, nz-1 that fall in this tile
          for (int q = threadIdx.x; q < 2 * S::TK + 2 * S::TJ; q += S::THREADS) {
            int j, k;
            if (q < 2 * S::TK) {
              j = q < S::TK ? 0 : a.ny - 1;
              k = k0 + (q % S::TK);
            } else {
              const int r = q - 2 * S::TK;
              k = r < S::TJ ? 0 : a.nz - 1;
              j = j0 + (r % S::TJ);
            }
            if (j < j0 || j >= j0 + S::TJ || j >= a.ny || k < k0 || k >= k0 + S::TK || k >= a.nz) continue;
            ge.emit(s, j, k, uc[(j - j0 + 2) * S::W + S::H + (k - k0)]);
          }
        }
      }
    }
    gbase += nload;
  }
}

// ---- host side --------------------------------------------------------------------------------

// View of a grid buffer for the sweep: x = k + H (base = row (i=-gx, j=-gy) at k = -H, which
// is pre-padding of that row), dims {nz+H+1, pny, pnx} so both z ghosts are inside and the last
// element of the view is inside the allocation (pnz >= nz + 2); box = one plane of the tile
// with its halos.
template <typename T>
ocu_status make_sweep_tmap(const void *buf, const ocu_layout &L, SweepTmap *out) {
  using S = SweepTile<T>;
  auto fn = encode_fn();
  if (!fn) return fail(OCU_ERR_CUDA, "[ERROR] cuTensorMapEncodeTiled is not available");
  const T *base = reinterpret_cast<const T *>(buf) +
                  (L.shift - (long long)L.gx * L.xstride - (long long)L.gy * L.ystride - S::H);
  cuuint64_t dims[3] = {(cuuint64_t)(L.nz + S::H + 1), (cuuint64_t)L.pny, (cuuint64_t)L.pnx};
  cuuint64_t strides[2] = {(cuuint64_t)L.ystride * sizeof(T), (cuuint64_t)L.xstride * sizeof(T)};
  cuuint32_t box[3] = {(cuuint32_t)S::W, (cuuint32_t)S::R, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  static_assert(sizeof(SweepTmap) == sizeof(CUtensorMap), "opaque tensor map size");
  CUresult r = fn(reinterpret_cast<CUtensorMap *>(out->bytes),
                  sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                  const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(OCU_ERR_CUDA, "[ERROR] cuTensorMapEncodeTiled failed (%d)", (int)r);
  return OCU_OK;
}

bool sweep2_supported(const ocu_layout &L, const ocu_bc_set &bc) {
  if (L.nz % 8 != 0 || L.nx < 2 || L.ny < 2 || L.nz < 8) return false;
  const ocu_bc *f[6] = {&bc.xpos, &bc.xneg, &bc.ypos, &bc.yneg, &bc.zpos, &bc.zneg};
  for (const ocu_bc *b : f)
    if (b->type != OCU_BC_DIRICHELET && b->type != OCU_BC_NEUMANN) return false;
  if (L.gx != 1 || L.gy != 1 || L.gz != 1) return false;
  if (L.pnz < L.nz + SweepTile<float>::H + 1) return false;
  return true;
}

// Resident CTAs per device (all SMs, shared-memory and register limits), computed once.
template <typename T>
static ocu_status sweep_slots(int *slots) {
  using S = SweepTile<T>;
  static int cache[64] = {0};
  static std::mutex mu;
  int dev = 0;
  OCU_TRY(check_cuda(cudaGetDevice(&dev), "cudaGetDevice"));
  std::lock_guard<std::mutex> lock(mu);
  if (!cache[dev & 63]) {
    OCU_TRY(check_cuda(cudaFuncSetAttribute(k_relax_sweep2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)S::SMEM),
                       "cudaFuncSetAttribute(k_relax_sweep2)"));
    int per_sm = 0, sms = 0;
    OCU_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_relax_sweep2<T>, S::THREADS, S::SMEM),
                       "cudaOccupancyMaxActiveBlocksPerMultiprocessor"));
    OCU_TRY(check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count"));
    if (per_sm < 1) return fail(OCU_ERR_CUDA, "[ERROR] k_relax_sweep2 does not fit on an SM");
    cache[dev & 63] = per_sm * sms;
  }
  *slots = cache[dev & 63];
  return OCU_OK;
}

template <typename T>
ocu_status launch_relax_sweep2(const SweepTmap &tm_u_in, const SweepTmap &tm_b, T *u_out, const ocu_layout &L,
                               const T *diag, int first_color, const RelaxParams &p, double hx, double hy, double hz,
                               int *err, cudaStream_t s, int wait_limit) {
  using S = SweepTile<T>;
  int slots = 0;
  OCU_TRY(sweep_slots<T>(&slots));
  SweepArgs a;
  a.nx = L.nx; a.ny = L.ny; a.nz = L.nz;
  a.gx = L.gx; a.gy = L.gy;
  a.first_color = first_color & 1;
  a.ntk = (L.nz + S::TK - 1) / S::TK;
  const int ntj = (L.ny + S::TJ - 1) / S::TJ;
  a.steps = (long long)a.ntk * ntj * L.nx;
  a.stall_test = wait_limit < 0;
  a.wait_limit = wait_limit < 0 ? -wait_limit : (wait_limit > 0 ? wait_limit : kWaitLimit);
  // one wave of resident CTAs, at least 8 plane steps each
  long long grid = a.steps / 8;
  if (grid > slots) grid = slots;
  if (grid < 1) grid = 1;
  const RelaxCoefD<T> c = make_relax_coef_d<T>(p);
  GhostEmit<T> ge{u_out, L.xstride, L.ystride, L.nx, L.ny, L.nz, to_dev(p.bc), (T)hx, (T)hy, (T)hz};
  CUtensorMap tu, tb;
  std::memcpy(&tu, tm_u_in.bytes, sizeof(tu));
  std::memcpy(&tb, tm_b.bytes, sizeof(tb));
  launch_pdl(k_relax_sweep2<T>, (unsigned)grid, S::THREADS, S::SMEM, s, tu, tb, u_out, L.xstride, L.ystride, a, c, diag,
             ge, err);
  return check_launch("k_relax_sweep2");
}

template ocu_status make_sweep_tmap<float>(const void *, const ocu_layout &, SweepTmap *);
template ocu_status make_sweep_tmap<double>(const void *, const ocu_layout &, SweepTmap *);
template ocu_status launch_relax_sweep2<float>(const SweepTmap &, const SweepTmap &, float *, const ocu_layout &,
                                               const float *, int, const RelaxParams &, double, double, double, int *,
                                               cudaStream_t, int);
template ocu_status launch_relax_sweep2<double>(const SweepTmap &, const SweepTmap &, double *, const ocu_layout &,
                                                const double *, int, const RelaxParams &, double, double, double,
                                                int *, cudaStream_t, int);

}  // namespace ocub
