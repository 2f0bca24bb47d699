/*
 * ocu_types.h -- plain-C value types shared by the C ABI (ocu_b200.h), the C++ facade
 * (include/ocu/) and the CPU oracle.
 *
 * Every enum value and struct field below is bit-compatible with the OpenCurrent type it
 * replaces, so a caller that fills the reference's structs can hand the same bytes across:
 *   ocu_bc_type / ocu_bc / ocu_bc_set  <- ocuutil/boundary_condition.h:26-112
 *   ocu_convergence                    <- ocuutil/convergence.h:27-40
 *   ocu_interpolation                  <- ocuutil/interpolation.h:26-31
 *   ocu_timestep                       <- ocuutil/timestep.h:28-32
 *   ocu_direction                      <- ocuutil/direction.h:26-39
 *   ocu_layout                         <- ocustorage/grid3d.h:29-96 + grid3ddev.cu:358-400
 */
#ifndef OCU_TYPES_H
#define OCU_TYPES_H

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary condition kinds (ocuutil/boundary_condition.h:26-36). */
typedef enum ocu_bc_type {
  OCU_BC_INVALID = 0,
  OCU_BC_NONE = 1,
  OCU_BC_PERIODIC = 2,
  OCU_BC_DIRICHELET = 3,
  OCU_BC_NEUMANN = 4,
  OCU_BC_SECOND_DERIV = 5,
  OCU_BC_DIRICHELET_AND_NEUMANN = 6,
  OCU_BC_FORCED_INFLOW_VARIABLE_SLIP = 7,
  OCU_BC_SCALAR_SLIP = 8
} ocu_bc_type;

/* One face's condition: the reference keeps value/aux_value as float
 * (ocuutil/boundary_condition.h:38-41), so do we. */
typedef struct ocu_bc {
  int type;          /* ocu_bc_type */
  float value;
  float aux_value;
} ocu_bc;

/* Six faces in the reference's member order (ocuutil/boundary_condition.h:62-64). */
typedef struct ocu_bc_set {
  ocu_bc xpos, xneg, ypos, yneg, zpos, zneg;
} ocu_bc_set;

/* Convergence flags (ocuutil/convergence.h:27-40). */
typedef enum ocu_convergence {
  OCU_CONVERGENCE_CALC_L2 = 0x01,
  OCU_CONVERGENCE_CALC_LINF = 0x02,
  OCU_CONVERGENCE_CRITERIA_L2 = 0x04,
  OCU_CONVERGENCE_CRITERIA_LINF = 0x08,
  OCU_CONVERGENCE_CRITERIA_NONE = 0x10,
  OCU_CONVERGENCE_L2 = 0x01 | 0x04,
  OCU_CONVERGENCE_LINF = 0x02 | 0x08,
  OCU_CONVERGENCE_NONE = 0x10,
  OCU_CONVERGENCE_NONE_CALC_L2LINF = 0x10 | 0x01 | 0x02
} ocu_convergence;

/* Preconditioners of the conjugate-gradient pressure solver (ocuequation/sol_pcgpressure3d.h:34-39). */
typedef enum ocu_precond {
  OCU_PRECOND_NONE = 0,
  OCU_PRECOND_JACOBI = 1,
  OCU_PRECOND_MULTIGRID = 2,
  OCU_PRECOND_BFBT = 3
} ocu_precond;

/* Grid staggering of a NetCDF grid variable (ocustorage/gridnetcdf.h:32-38). */
typedef enum ocu_grid_staggering {
  OCU_GS_CENTER_POINT = 0,
  OCU_GS_U_FACE = 1,
  OCU_GS_V_FACE = 2,
  OCU_GS_W_FACE = 3,
  OCU_GS_CUSTOM = 4
} ocu_grid_staggering;

/* Value types of NetCDF variables (the netCDF library's nc_type codes). */
typedef enum ocu_nc_type { OCU_NC_INT = 4, OCU_NC_FLOAT = 5, OCU_NC_DOUBLE = 6 } ocu_nc_type;

/* Advection interpolants (ocuutil/interpolation.h:26-31). */
typedef enum ocu_interpolation {
  OCU_IT_ERROR = 0,
  OCU_IT_FIRST_ORDER_UPWIND = 1,
  OCU_IT_SECOND_ORDER_CENTERED = 2,
  OCU_IT_THIRD_ORDER_VAN_LEER_FLUX_LIMITED = 3
} ocu_interpolation;

/* Time integrators (ocuutil/timestep.h:28-32). */
typedef enum ocu_timestep {
  OCU_TS_ERROR = 0,
  OCU_TS_FORWARD_EULER = 1,
  OCU_TS_ADAMS_BASHFORD2 = 2
} ocu_timestep;

/* Axis/direction flags (ocuutil/direction.h:26-39). */
typedef enum ocu_direction {
  OCU_DIR_POSITIVE_FLAG = 0x01,
  OCU_DIR_NEGATIVE_FLAG = 0x02,
  OCU_DIR_XAXIS_FLAG = 0x04,
  OCU_DIR_YAXIS_FLAG = 0x08,
  OCU_DIR_ZAXIS_FLAG = 0x10,
  OCU_DIR_XPOS = 0x04 | 0x01,
  OCU_DIR_XNEG = 0x04 | 0x02,
  OCU_DIR_YPOS = 0x08 | 0x01,
  OCU_DIR_YNEG = 0x08 | 0x02,
  OCU_DIR_ZPOS = 0x10 | 0x01,
  OCU_DIR_ZNEG = 0x10 | 0x02
} ocu_direction;

/* Element type of a grid. */
typedef enum ocu_dtype {
  OCU_F32 = 0,
  OCU_F64 = 1
} ocu_dtype;

/*
 * Padded, z-fastest storage of a cell grid with ghost layers -- the Grid3DDevice<T> memory
 * contract (ocustorage/grid3d.h:29-96, grid3ddev.cu:358-400):
 *   pnx = nx + 2gx + padx, pny = ny + 2gy + pady,
 *   pnz = nz + 2gz + padz rounded up to a multiple of 16,
 *   element (i,j,k) lives at  shift + i*xstride + j*ystride + k,  i,j,k in [-g, n+g),
 *   shift = gx*xstride + gy*ystride + 16  (16-gz elements of pre-padding put k=0 of every
 *   row on a 16-element boundary),
 *   allocated = pnx*pny*pnz + 16 - gz.
 */
typedef struct ocu_layout {
  int nx, ny, nz;
  int gx, gy, gz;
  int pnx, pny, pnz;
  int xstride, ystride;
  long long shift;
  long long allocated;
} ocu_layout;

/* Reduction operators of Grid3DDevice<T>::reduce_* (ocustorage/grid3d.h:237-242). */
typedef enum ocu_reduce_op {
  OCU_REDUCE_MAXABS = 0,
  OCU_REDUCE_MAX = 1,
  OCU_REDUCE_MIN = 2,
  OCU_REDUCE_SUM = 3,
  OCU_REDUCE_SQRSUM = 4,
  OCU_REDUCE_CHECKNAN = 5
} ocu_reduce_op;

/* Ghost-fill variants of ocustorage/grid3dboundary.h:26-70. */
typedef enum ocu_bc_variant {
  OCU_BC_LEVEL1 = 0,            /* faces, edges and corners: apply_3d_boundary_conditions_level1 */
  OCU_BC_LEVEL1_NOCORNERS = 1   /* faces only: apply_3d_boundary_conditions_level1_nocorners */
} ocu_bc_variant;

#ifdef __cplusplus
}
#endif

#endif /* OCU_TYPES_H */
