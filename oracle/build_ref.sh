#!/usr/bin/env bash
# TEST INFRASTRUCTURE ONLY.  Compiles the reference's generic_simple_v1 sources where they lie
# under /root/reference (nothing is copied into this repository) together with this directory's
# single-rank MPI / HYPRE stand-ins (ref_stubs/).  Outputs, all under oracle/_ref/ (git-ignored):
#   libgsv1ref.so  ref_shim.cu (#includes the reference main.cu) + the reference BC sources
#   gsv1_ref       the reference program itself (its main()), for end-to-end runs on a GPU box
#   libscalarref.so  the reference's libpoisson / libscalar host assembly (ref_scalar_shim.cu,
#                    ref_transport_shim.cu)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
SRC=/root/reference/apps/generic_simple_v1/src
OUT="$HERE/_ref"
NVCC="${CUDA_HOME:-/usr/local/cuda}/bin/nvcc"
mkdir -p "$OUT"
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -I"$HERE/ref_stubs" -I"$SRC"
       -Xcompiler -fPIC,-ffp-contract=off -w)
BC=("$SRC/bc_specs.cu" "$SRC/bc_runtime_config.cu" "$SRC/velocity_bc_eval.cu" "$SRC/patch_geometry.cu")
for f in "${BC[@]}"; do
  "$NVCC" "${FLAGS[@]}" -c "$f" -o "$OUT/$(basename "$f" .cu).o"
done
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_stubs/mini_hypre.cu" -o "$OUT/mini_hypre.o"
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_shim.cu" -o "$OUT/ref_shim.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libgsv1ref.so" "$OUT/ref_shim.o" \
  "$OUT/mini_hypre.o" "$OUT"/bc_specs.o "$OUT"/bc_runtime_config.o "$OUT"/velocity_bc_eval.o "$OUT"/patch_geometry.o
"$NVCC" "${FLAGS[@]}" -c "$SRC/main.cu" -o "$OUT/gsv1_main.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -o "$OUT/gsv1_ref" "$OUT/gsv1_main.o" "$OUT/mini_hypre.o" \
  "$OUT"/bc_specs.o "$OUT"/bc_runtime_config.o "$OUT"/velocity_bc_eval.o "$OUT"/patch_geometry.o

# libscalarref.so: the reference's libpoisson mesh reader / gradient / elliptic assembly
# (ref_scalar_shim.cu) and libscalar's transport assembly (ref_transport_shim.cu includes
# scalar_transport_library.cu)
PS=/root/reference/libpoisson
LS=/root/reference/libscalar
SFLAGS=(-gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -I"$HERE/ref_stubs" -I"$PS/include"
        -I"$LS/include" -I"$LS/src" -Xcompiler -fPIC,-ffp-contract=off -w)
for f in mesh gradient scalar_elliptic bc; do
  "$NVCC" "${SFLAGS[@]}" -c "$PS/src/$f.cu" -o "$OUT/ps_$f.o"
done
"$NVCC" "${SFLAGS[@]}" -c "$HERE/ref_scalar_shim.cu" -o "$OUT/ref_scalar_shim.o"
"$NVCC" "${SFLAGS[@]}" -c "$HERE/ref_transport_shim.cu" -o "$OUT/ref_transport_shim.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libscalarref.so" "$OUT/ref_scalar_shim.o" \
  "$OUT/ref_transport_shim.o" \
  "$OUT"/ps_mesh.o "$OUT"/ps_gradient.o "$OUT"/ps_scalar_elliptic.o "$OUT"/ps_bc.o "$OUT/mini_hypre.o"
rm -f "$OUT"/*.o
echo "$OUT/libgsv1ref.so"
