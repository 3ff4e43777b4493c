#!/bin/bash
# Builds the reference code itself as a CPU oracle / CPU baseline:
# GIZMO's own sources, read where they lie in the reference tree, compiled
# against project-written single-rank MPI and minimal GSL stand-ins (shim/)
# and linked with ref_main.c instead of main.c.  Output: oracle/_ref/gizmo_ref.
# Nothing from the reference tree is copied into the repository: the compile
# reads a symlink mirror under a temporary directory, needed only so that the
# reference's relative include of ../GIZMO_config.h resolves to shim/GIZMO_config.h.
# TEST INFRASTRUCTURE ONLY.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${GIZMO_REF:-/root/reference}"
OUT="$HERE/_ref"
CC=/usr/bin/gcc
# x86-64-v3 (AVX2/FMA): the binary runs on the GPU hosts as well as here
CFLAGS="-O3 -march=x86-64-v3 -fopenmp -std=gnu99 -w"
if [ ! -d "$REF" ]; then echo "reference tree not found: $REF" >&2; exit 1; fi
if [ -x "$OUT/gizmo_ref" ] && [ -x "$OUT/gizmo_ref_pot" ] && [ -x "$OUT/gizmo_b200" ] && [ "$OUT/gizmo_b200" -nt "$HERE/ref_main.c" ] && [ "$OUT/gizmo_b200" -nt "$0" ] && [ "$OUT/gizmo_b200" -nt "$HERE/../gizmo-public_b200/host/gravtree_b200.c" ] && [ "$OUT/gizmo_b200" -nt "$HERE/../include/gizmo_gravity_b200.h" ] && [ "$OUT/gizmo_b200" -nt "$HERE/patch_gravtree.py" ] && [ "$OUT/gizmo_ref_pot" -nt "$HERE/ref_main.c" ]; then
  echo "oracle/_ref/gizmo_ref is up to date"; exit 0
fi
MIRROR="$(mktemp -d /tmp/gg_ref_src.XXXXXX)"
trap 'rm -rf "$MIRROR"' EXIT
cp -rs "$REF/." "$MIRROR/"
cp "$HERE/shim/GIZMO_config.h" "$MIRROR/GIZMO_config.h"
mkdir -p "$OUT/obj"
cd "$MIRROR"
# the object list of the reference Makefile (CORE..MISC groups) without main.o
# and the generated compile_time_info.o
FILES="accel.c timestep.c init.c restart.c io.c predict.c global.c begrun.c run.c allvars.c read_ic.c domain.c
driftfac.c kicks.c ngb.c merge_split.c system/system.c system/allocate.c system/mymalloc.c system/parallel_sort.c
system/peano.c system/parallel_sort_special.c system/mpi_util.c system/pinning.c gravity/forcetree.c
gravity/forcetree_update.c gravity/gravtree.c gravity/cosmology.c gravity/potential.c gravity/pm_periodic.c
gravity/pm_nonperiodic.c gravity/longrange.c gravity/ags_hsml.c gravity/binary.c hydro/hydro_toplevel.c
hydro/density.c hydro/gradients.c turb/dynamic_diffusion.c turb/dynamic_diffusion_velocities.c turb/turb_driving.c
turb/turb_powerspectra.c cooling/cooling.c cooling/grackle.c eos/eos.c eos/hydrogen_molecule.c
eos/cosmic_ray_fluid/cosmic_ray_alfven.c eos/cosmic_ray_fluid/cosmic_ray_utilities.c solids/elastic_physics.c
solids/grain_physics.c solids/ism_dust_chemistry.c nuclear/nuclear_network_solver.c nuclear/nuclear_network.c
galaxy_sf/sfr_eff.c galaxy_sf/stellar_evolution.c galaxy_sf/mechanical_fb.c galaxy_sf/thermal_fb.c
galaxy_sf/radfb_local.c galaxy_sf/dm_dispersion_hsml.c galaxy_sf/blackholes/blackhole.c
galaxy_sf/blackholes/blackhole_util.c galaxy_sf/blackholes/blackhole_environment.c galaxy_sf/blackholes/blackhole_feed.c
galaxy_sf/blackholes/blackhole_swallow_and_kick.c radiation/rt_utilities.c radiation/rt_CGmethod.c
radiation/rt_source_injection.c radiation/rt_chem.c radiation/rt_cooling.c structure/fof.c structure/subfind/subfind.c
structure/subfind/subfind_vars.c structure/subfind/subfind_collective.c structure/subfind/subfind_serial.c
structure/subfind/subfind_so.c structure/subfind/subfind_cont.c structure/subfind/subfind_distribute.c
structure/subfind/subfind_findlinkngb.c structure/subfind/subfind_nearesttwo.c structure/subfind/subfind_loctree.c
structure/subfind/subfind_potential.c structure/subfind/subfind_density.c structure/twopoint.c structure/lineofsight.c
sidm/cbe_integrator.c sidm/dm_fuzzy.c sidm/sidm_core.c"
OBJS=""
for f in $FILES; do
  o="$OUT/obj/$(echo "$f" | tr / _ | sed 's/\.c$/.o/')"
  OBJS="$OBJS $o"
  echo "$CC $CFLAGS -I$HERE/shim -I$MIRROR -c $f -o $o"
done > "$MIRROR/cmds.sh"
xargs -P "$(nproc)" -I{} bash -c '{}' < "$MIRROR/cmds.sh"
$CC $CFLAGS -I"$HERE/shim" -I"$MIRROR" -c "$HERE/ref_main.c" -o "$OUT/obj/ref_main.o"
$CC $CFLAGS -I"$HERE/shim" -c "$HERE/shim/mpi_single.c" -o "$OUT/obj/mpi_single.o"
$CC $CFLAGS -I"$HERE/shim" -c "$HERE/shim/gsl_shim.c" -o "$OUT/obj/gsl_shim.o"
$CC $CFLAGS -o "$OUT/gizmo_ref" $OBJS "$OUT/obj/ref_main.o" "$OUT/obj/mpi_single.o" "$OUT/obj/gsl_shim.o" -lm
echo "built $OUT/gizmo_ref"
# variant without EVALPOTENTIAL, with COMPUTE_POTENTIAL_ENERGY: it has the
# separate potential-only walk (compute_potential) that the harness calls
# after the start-up passes.  Output: oracle/_ref/gizmo_ref_pot.
MIRROR_POT="$MIRROR/pot_tree"
mkdir -p "$MIRROR_POT"
cp -rs "$REF/." "$MIRROR_POT/"
rm -f "$MIRROR_POT/GIZMO_config.h"
cp "$HERE/shim/pot/GIZMO_config.h" "$MIRROR_POT/GIZMO_config.h"
mkdir -p "$OUT/obj_pot"
OBJS_POT=""
for f in $FILES; do
  o="$OUT/obj_pot/$(echo "$f" | tr / _ | sed 's/\.c$/.o/')"
  OBJS_POT="$OBJS_POT $o"
  echo "cd $MIRROR_POT && $CC $CFLAGS -I$HERE/shim -I$MIRROR_POT -c $f -o $o"
done > "$MIRROR/cmds_pot.sh"
xargs -P "$(nproc)" -I{} bash -c '{}' < "$MIRROR/cmds_pot.sh"
$CC $CFLAGS -DGG_WITH_COMPUTE_POTENTIAL -I"$HERE/shim" -I"$MIRROR_POT" -c "$HERE/ref_main.c" -o "$OUT/obj_pot/ref_main.o"
$CC $CFLAGS -o "$OUT/gizmo_ref_pot" $OBJS_POT "$OUT/obj_pot/ref_main.o" "$OUT/obj/mpi_single.o" "$OUT/obj/gsl_shim.o" -lm
echo "built $OUT/gizmo_ref_pot"
# GIZMO driving the B200 library: the reference's own gravity/gravtree.c with
# the GRAVITY_GPU_B200 blocks of INTEGRATION.md added by patch_gravtree.py
# (written into a third mirror, over its symlink), compiled with
# -DGRAVITY_GPU_B200 and linked with the C host code
# (gizmo-public_b200/host/gravtree_b200.c) and the CUDA library
PKG="$(cd "$HERE/../gizmo-public_b200" && pwd)"
if [ -f "$PKG/libgizmo_gravity_b200.so" ]; then
  MIRROR_B200="$MIRROR/b200_tree"
  mkdir -p "$MIRROR_B200"
  cp -rs "$REF/." "$MIRROR_B200/"
  rm -f "$MIRROR_B200/GIZMO_config.h"
  cp "$HERE/shim/GIZMO_config.h" "$MIRROR_B200/GIZMO_config.h"
  python3 "$HERE/patch_gravtree.py" "$REF/gravity/gravtree.c" "$MIRROR_B200/gravity/gravtree.c"
  (cd "$MIRROR_B200" && $CC $CFLAGS -DGRAVITY_GPU_B200 -I"$HERE/shim" -I"$MIRROR_B200" -c gravity/gravtree.c \
      -o "$OUT/obj/gravity_gravtree_b200.o")
  OBJS_B200="$(echo $OBJS | tr ' ' '\n' | grep -v '/gravity_gravtree\.o$' | tr '\n' ' ')"
  $CC $CFLAGS -DGG_USE_B200 -I"$HERE/shim" -I"$MIRROR" -c "$HERE/ref_main.c" -o "$OUT/obj/ref_main_b200.o"
  $CC $CFLAGS -I"$HERE/shim" -I"$MIRROR" -I"$PKG/../include" -c "$PKG/host/gravtree_b200.c" -o "$OUT/obj/gravtree_b200.o"
  $CC $CFLAGS -o "$OUT/gizmo_b200" $OBJS_B200 "$OUT/obj/gravity_gravtree_b200.o" "$OUT/obj/ref_main_b200.o" \
      "$OUT/obj/gravtree_b200.o" "$OUT/obj/mpi_single.o" "$OUT/obj/gsl_shim.o" -L"$PKG" -lgizmo_gravity_b200 \
      -Wl,-rpath,'$ORIGIN/../../gizmo-public_b200' -lm
  echo "built $OUT/gizmo_b200"
fi
