#!/usr/bin/env bash
# Build oracle/_ref/libpiny_ref.so from the reference's own PINY physics
# sources (read in place under /root/reference; nothing is copied) plus the
# project-written stubs in oracle/ref_stubs and oracle/ref_shim.C.
# Test infrastructure only.  Output stays in oracle/_ref/ (git-ignored).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${OA_REFERENCE:-/root/reference}"
PINY="$REF/src_piny_physics_v1.0"
OUT="$HERE/_ref"
if [ ! -d "$PINY" ]; then echo "reference tree not found at $REF; skipping oracle/_ref" >&2; exit 0; fi
mkdir -p "$OUT"
CXX="${CXX:-g++}"
FLAGS="-O2 -fPIC -std=c++14 -DCHARM_ON -DFORTRANUNDERSCORE -w -include $HERE/ref_stubs/charm++.h -I$HERE/ref_stubs -I$PINY/include/pentium -I$PINY/include -I$REF/src_mathlib -I$REF/include"
SRCS=(
  "$PINY/abinito_physics/cp_nonlocal/cp_eke.C"
  "$PINY/abinito_physics/cp_xc_fnctl/cp_pz_lda.C"
  "$PINY/abinito_physics/cp_xc_fnctl/cp_becke.C"
  "$PINY/abinito_physics/cp_xc_fnctl/cp_grad_rho_ctrl.C"
  "$PINY/abinito_physics/cp_local/cp_hart_ext.C"
  "$PINY/abinito_physics/cp_orthog/cp_lowdin.C"
  "$PINY/abinito_physics/cp_nonlocal/cp_struct_fact.C"
  "$PINY/abinito_physics/cp_nonlocal/cp_nlmat.C"
  "$PINY/abinito_physics/cp_nonlocal/cp_nl_energy_forc.C"
  "$PINY/abinito_physics/cp_integrate/cp_dynamics.C"
  "$PINY/abinito_physics/cp_integrate/cp_isokin.C"
  "$PINY/abinito_physics/cp_integrate/cp_min_std.C"
  "$PINY/abinito_physics/cp_integrate/cp_min_CG.C"
  "$PINY/abinito_physics/cp_nonlocal/cp_ees_nonlocal.C"
  "$PINY/interface/cp_ewald/set_cp_ewald.C"
  "$PINY/abinito_physics/cp_ions/cp_rspace_ion.C"
  "$PINY/interface/vps_params/control_vps_params.C"
  "$PINY/friend_lib/friend_lib.C"
)
OBJS=()
for s in "${SRCS[@]}"; do
  o="$OUT/$(basename "$s" .C).o"
  $CXX $FLAGS -c "$s" -o "$o"
  OBJS+=("$o")
done
# the shim sits beside the PINY sources' include layout via -iquote
$CXX $FLAGS -iquote "$PINY/abinito_physics/cp_local" -c "$HERE/ref_shim.C" -o "$OUT/ref_shim.o"
$CXX -shared -Wl,--no-undefined -o "$OUT/libpiny_ref.so" "${OBJS[@]}" "$OUT/ref_shim.o"
echo "$OUT/libpiny_ref.so"
