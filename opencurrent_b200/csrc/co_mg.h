// Multi-image multigrid (Sol_MultigridPressure3DDeviceCo, sol_mgpressure3d.h:184-242,
// sol_mgpressure3dco.cu:39-529): the interface the driver of mg_solver.cu sees.
#pragma once

#include <memory>
#include <vector>

#include "ocu_internal.h"

namespace ocub {

struct CoreOps;

// The level operations of a multi-image hierarchy plus what only it has.
struct CoOps {
  virtual ~CoOps() {}
  virtual CoreOps *ops() = 0;
  virtual ocu_grid *pressure(int image) = 0;
  virtual int images() const = 0;
  virtual int cutoff_level() const = 0;
  virtual const int *coarse_dim() const = 0;  // global dimensions of the coarsest level
};

// Host-side decomposition of one image (sol_mgpressure3dco.cu:242-300, 420-435): the level count
// of the global hierarchy, the cutoff level (the first level >= 1 whose global cell count is at
// most cutoff_cells; levels from there on are held whole by image 0), the x neighbours (-1 at a
// face of the domain; periodic x wraps) and the image's faces at level 0 (BC_NONE where a
// neighbour's plane is copied in).
ocu_status mgco_plan(int nx_local, int ny, int nz, int num_images, int image, long long cutoff_cells,
                     const ocu_bc_set &bc, ocu_mgco_plan *out);

// Builds the hierarchy of `num_images` slabs of nx_local x ny x nz (rhs[i] on devices[i]).
// pressure0: image 0's level-0 u, allocated by the caller with rhs[0]'s layout.
ocu_status mgco_create(ocu_dtype dt, int num_images, const int *devices, int nx_local, int ny, int nz, double hx,
                       double hy, double hz, ocu_grid *const *rhs, ocu_grid *pressure0, const ocu_mg_params &prm,
                       long long cutoff_cells, cudaStream_t stream0, std::unique_ptr<CoOps> *out);

}  // namespace ocub
