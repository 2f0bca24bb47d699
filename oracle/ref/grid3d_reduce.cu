/*
 * grid3d_reduce.cu -- TEST INFRASTRUCTURE ONLY (linked into oracle/_ref by build_ref.sh in
 * place of ocustorage/grid3dops.cu).
 *
 * ocustorage/grid3dops.cu:26-130 reduces a Grid3DDevice in two stages: one warp per (i,j)
 * row folds k, k+32, k+64, ... per lane, then a 16/8/4/2/1 tree over the 32 lanes, written
 * warp-synchronously through plain shared memory with neither volatile nor __syncwarp
 * (grid3dops.cu:74-82).  Since sm_70 lanes are not guaranteed to run in lock step and the
 * compiler may reorder those shared loads and stores, so the as-shipped kernel can return a
 * wrong norm on a B200.  This file supplies the same entry point with the same fold order
 * (per-lane strided fold in the same order, the same tree pairs, the same 2x2 (i,j) blocks
 * and the same 1-D second stage, ocustorage/grid1dops.cu) with the tree done by warp
 * shuffles, which are synchronous by definition.  Nothing else of the reference is changed.
 */
#include <cstdio>

#include "ocustorage/grid1dops.h"
#include "ocustorage/grid3dops.h"
#include "ocuutil/reduction_op.h"
#include "ocuutil/thread.h"

template <typename T, typename REDUCE>
__global__ void ref_row_fold(T *grid2d, int xstride2d, const T *grid, int xstride, int ystride,
                             int nx, int ny, int nz, REDUCE red) {
  /* blockDim = (32, 2, 2): x is the lane along k, z picks i, y picks j (grid3dops.cu:33-37) */
  int i = blockIdx.x * blockDim.z + threadIdx.z;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return; /* uniform over the warp: all its lanes share (i, j) */
  const T *row = grid + xstride * i + ystride * j;
  T acc = red.identity();
  int k = threadIdx.x;
  if (k < nz) acc = red.process(row[k]);
  for (k += 32; k < nz; k += 32) acc = red.reduce(red.process(row[k]), acc);
  for (int s = 16; s >= 1; s >>= 1) {
    T other = __shfl_down_sync(0xffffffffu, acc, s);
    if ((int)threadIdx.x < s) acc = red.reduce(acc, other);
  }
  if (threadIdx.x == 0) grid2d[i * xstride2d + j] = acc;
}

namespace ocu {

template <typename T, typename REDUCE>
bool reduce_with_operator(const ocu::Grid3DDevice<T> &grid, T &result, REDUCE reduce) {
  ocu::Grid1DDevice<T> rows;
  rows.init(grid.nx() * grid.ny(), 0);
  dim3 Dg((grid.nx() + 1) / 2, (grid.ny() + 1) / 2);
  dim3 Db(32, 2, 2);
  ref_row_fold<<<Dg, Db, 0, ThreadManager::get_compute_stream()>>>(
      &rows.at(0), grid.ny(), &grid.at(0, 0, 0), grid.xstride(), grid.ystride(), grid.nx(),
      grid.ny(), grid.nz(), reduce);
  cudaError_t er = cudaGetLastError();
  if (er != cudaSuccess) {
    printf("[ERROR] reduce_with_operator - row fold failed: %s\n", cudaGetErrorString(er));
    return false;
  }
  if (!reduce_with_operator(rows, result, reduce, true)) {
    printf("[ERROR] reduce_with_operator - 1d reduction failed\n");
  }
  return true;
}

template bool reduce_with_operator(const Grid3DDevice<float> &, float &, ReduceDevMaxF);
template bool reduce_with_operator(const Grid3DDevice<float> &, float &, ReduceDevMinF);
template bool reduce_with_operator(const Grid3DDevice<float> &, float &, ReduceDevMaxAbsF);
template bool reduce_with_operator(const Grid3DDevice<float> &, float &, ReduceDevSum<float>);
template bool reduce_with_operator(const Grid3DDevice<float> &, float &, ReduceDevSqrSum<float>);
template bool reduce_with_operator(const Grid3DDevice<float> &, float &, ReduceDevCheckNan<float>);
template bool reduce_with_operator(const Grid3DDevice<int> &, int &, ReduceDevMaxI);
template bool reduce_with_operator(const Grid3DDevice<int> &, int &, ReduceDevMinI);
template bool reduce_with_operator(const Grid3DDevice<int> &, int &, ReduceDevMaxAbsI);
template bool reduce_with_operator(const Grid3DDevice<int> &, int &, ReduceDevSum<int>);
template bool reduce_with_operator(const Grid3DDevice<int> &, int &, ReduceDevSqrSum<int>);
template bool reduce_with_operator(const Grid3DDevice<double> &, double &, ReduceDevMaxD);
template bool reduce_with_operator(const Grid3DDevice<double> &, double &, ReduceDevMinD);
template bool reduce_with_operator(const Grid3DDevice<double> &, double &, ReduceDevMaxAbsD);
template bool reduce_with_operator(const Grid3DDevice<double> &, double &, ReduceDevSum<double>);
template bool reduce_with_operator(const Grid3DDevice<double> &, double &, ReduceDevSqrSum<double>);
template bool reduce_with_operator(const Grid3DDevice<double> &, double &, ReduceDevCheckNan<double>);

}  // namespace ocu
