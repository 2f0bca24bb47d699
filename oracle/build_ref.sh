#!/usr/bin/env bash
# build_ref.sh -- TEST INFRASTRUCTURE ONLY.
#
# Compiles OpenCurrent's own device solver, from the reference sources where they lie, into
# oracle/_ref/libocu_ref.so (git-ignored; it travels with the tree to GPU machines), for the
# GPU parity tests that compare the B200 library with the reference on identical inputs.
#
#   bash oracle/build_ref.sh [REFERENCE_ROOT]      (default: /root/reference)
#
# Nothing is copied out of the reference tree.  Two things are added around it:
#   oracle/ref/texture_shim.h   force-included: CUDA 12 removed the legacy texture references
#                               used by sol_mgpressure3ddevf.cu, sol_mgpressure3ddevd.cu and
#                               sol_selfadvection3ddev.cu; the shim reads the same buffers
#                               through __ldg.
#   oracle/ref/grid3d_reduce.cu replaces ocustorage/grid3dops.cu, whose warp stage is
#                               warp-synchronous without __syncwarp (undefined since sm_70);
#                               same fold order, done with shuffles.
#   oracle/ref/ref_driver.cu    a C entry layer over the reference classes for ctypes.
# Device code is built the way the reference's CMake built it (nvcc defaults, so a*b+c may
# be contracted to an FMA), for sm_100a; host code with g++ defaults (no -O, no FMA).
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-/root/reference}"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
LIB="$OUT/libocu_ref.so"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"

if [ ! -d "$REF/ocuequation" ]; then
  echo "build_ref.sh: reference tree not found at $REF; nothing built" >&2
  exit 1
fi

SOURCES=(
  ocuutil/kernel_wrapper.cu ocuutil/thread.cu ocuutil/memory.cu ocuutil/timer.cu
  ocuutil/timing_pool.cpp ocuutil/imagefile.cpp
  ocustorage/grid1ddev.cu ocustorage/grid1dhost.cu ocustorage/grid1dops.cu
  ocustorage/grid3ddev.cu ocustorage/grid3dhost.cu ocustorage/grid3d.cpp
  ocustorage/grid3dops.cpp ocustorage/grid3dboundary.cu ocustorage/grid2ddev.cu
  ocustorage/grid2dhost.cpp ocustorage/grid2dhost.cu ocustorage/coarray.cu
  ocustorage/transfer_q.cu ocustorage/transfer_routines.cu ocustorage/barrier_exchange.cu
  ocustorage/exchange_mempool.cu ocuequation/sol_mgpressure3dco.cu
  ocuequation/solver.cu ocuequation/equation.cpp ocuequation/eqn_incompressns3d.cu
  ocuequation/sol_passiveadvection3ddev.cu ocuequation/sol_selfadvection3ddev.cu
  ocuequation/sol_mgpressure3d.cpp ocuequation/sol_mgpressuremixed3ddevd.cpp
  ocuequation/sol_mgpressure3ddev.cu ocuequation/sol_mgpressure3ddevd.cu
  ocuequation/sol_mgpressure3ddevf.cu ocuequation/sol_project3ddev.cu
  ocuequation/sol_projectmixed3d.cu ocuequation/sol_project3d.cpp
  ocuequation/sol_laplaciancent3ddev.cu ocuequation/sol_divergence3ddev.cu
  ocuequation/sol_gradient3ddev.cu ocuequation/sol_pcgpressure3d.cu
)
LOCAL=(grid3d_reduce.cu ref_driver.cu)

FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++14 -Xcompiler -fPIC
       -I"$REF" -include "$HERE/ref/texture_shim.h"
       -DOCU_DOUBLESUPPORT -DOCU_ATOMICSUPPORT -DOCU_SM20 -w)

mkdir -p "$OBJ"
newest_dep=$(stat -c %Y "$HERE/ref/"* "$HERE/ocu_oracle.h" "$HERE/../include/ocu_types.h" \
             "$0" | sort -n | tail -1)

compile() {  # $1 = source path, $2 = object path
  local src="$1" obj="$2"
  if [ -f "$obj" ] && [ "$(stat -c %Y "$obj")" -gt "$(stat -c %Y "$src")" ] \
     && [ "$(stat -c %Y "$obj")" -gt "$newest_dep" ]; then
    return 0
  fi
  "$NVCC" "${FLAGS[@]}" -x cu -c "$src" -o "$obj"
}

pids=()
objs=()
for s in "${SOURCES[@]}"; do
  o="$OBJ/$(echo "$s" | tr '/' '_').o"
  objs+=("$o")
  compile "$REF/$s" "$o" & pids+=($!)
done
for s in "${LOCAL[@]}"; do
  o="$OBJ/local_${s}.o"
  objs+=("$o")
  compile "$HERE/ref/$s" "$o" & pids+=($!)
done
fail=0
for p in "${pids[@]}"; do wait "$p" || fail=1; done
if [ "$fail" -ne 0 ]; then
  echo "build_ref.sh: compilation failed" >&2
  exit 1
fi

"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$LIB.tmp" "${objs[@]}" \
  -lcudart_static -Xlinker --no-undefined
mv "$LIB.tmp" "$LIB"
echo "$LIB"
