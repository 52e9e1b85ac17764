#!/usr/bin/env bash
# Compiles LeonardYM's own fermion hot path from its sources under /root/reference
# (never copied into this repository) against the Eigen-API shim in
# oracle/eigen_shim, plus oracle/ref_harness.cpp, into oracle/_ref/:
#   libleonard_ref_su3.so     NUMCOLORS=3            (SU(3) fundamental)
#   libleonard_ref_su2adj.so  NUMCOLORS=2 -DADJOINT  (SU(2) adjoint)
#   libleonard_ref_su3_native.so  the SU(3) build again with -march=native (the CPU
#                             baseline of bench.py; the two builds above, for any x86-64,
#                             pin the oracle and make the golden fixtures)
# Flags follow the reference's Makefile.mth (-DEIGEN -DMULTITHREADING -fopenmp, the
# MatrixBase plugin) and Makefile.mpi (-march=native, native build only), with
# -std=c++17 because program_options uses <any>.  -march=native targets the CPU of the
# machine that runs this script; bench.py runs the native build only after a probe of it
# on the host that runs the benchmark succeeds.
set -euo pipefail
REF=${LYM_REFERENCE:-/root/reference}/source
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -d "$REF" ]; then
  # --if-present: a machine without the reference sources keeps the prebuilt oracle/_ref
  [ "${1:-}" = "--if-present" ] && { echo "reference sources absent: oracle/_ref kept as it is"; exit 0; }
  echo "reference sources not found at $REF" >&2; exit 1
fi
TUS=(
  MPILattice/LocalLayout.cpp
  dirac_operators/DiracOperator.cpp dirac_operators/DiracWilsonOperator.cpp
  dirac_operators/BasicDiracWilsonOperator.cpp dirac_operators/BasicSquareDiracWilsonOperator.cpp
  dirac_operators/ImprovedDiracWilsonOperator.cpp dirac_operators/EvenOddImprovedDiracWilsonOperator.cpp
  dirac_operators/SquareDiracWilsonOperator.cpp dirac_operators/SquareImprovedDiracWilsonOperator.cpp
  dirac_operators/SquareEvenOddImprovedDiracWilsonOperator.cpp
  dirac_operators/OverlapOperator.cpp dirac_operators/SquareOverlapOperator.cpp dirac_operators/ExactOverlapOperator.cpp
  dirac_functions/Polynomial.cpp dirac_functions/ChebyshevRecursion.cpp fermion_measurements/DiracEigenSolver.cpp
  dirac_functions/RationalApproximation.cpp
  inverters/ConjugateGradient.cpp inverters/BiConjugateGradient.cpp inverters/PreconditionedBiCGStab.cpp
  inverters/MultishiftSolver.cpp inverters/MEMultishiftSolver.cpp inverters/MMMRMultishiftSolver.cpp
  inverters/ChronologicalMultishiftSolver.cpp
  algebra_utils/AlgebraUtils.cpp utils/RandomSeed.cpp utils/Gamma.cpp
  program_options/StorageParameters.cpp
  hmc_forces/Force.cpp hmc_forces/FermionForce.cpp hmc_forces/DiracWilsonFermionForce.cpp
  hmc_forces/ImprovedFermionForce.cpp hmc_forces/OverlapFermionForce.cpp
  correlators/MesonCorrelator.cpp fermion_measurements/ChiralCondensate.cpp
  fermion_measurements/StochasticEstimator.cpp dirac_operators/Propagator.cpp io/GlobalOutput.cpp
  utils/StoutSmearing.cpp actions/WilsonGaugeAction.cpp actions/GaugeAction.cpp actions/ImprovedGaugeAction.cpp
  wilson_loops/Plaquette.cpp actions/Energy.cpp hmc_forces/GaugeForce.cpp
  starters/ReadStartGaugeConfiguration.cpp io/OutputSweep.cpp Environment.cpp
)
build() {
  local name=$1; shift
  local flags=("$@")
  local objdir="$OUT/obj_$name"
  mkdir -p "$objdir"
  local objs=()
  for tu in "${TUS[@]}" ; do
    local o="$objdir/$(echo "$tu" | tr '/' '_' | sed 's/\.cpp$/.o/')"
    if [ ! -f "$o" ] || [ "$REF/$tu" -nt "$o" ] || [ "$HERE/eigen_shim/Eigen/Dense" -nt "$o" ] || [ "$HERE/build_ref.sh" -nt "$o" ]; then
      g++ "${flags[@]}" -c "$REF/$tu" -o "$o" &
    fi
    objs+=("$o")
  done
  wait
  g++ "${flags[@]}" -c "$HERE/ref_harness.cpp" -o "$objdir/ref_harness.o"
  g++ "${flags[@]}" -c "$HERE/ref_stubs.cpp" -o "$objdir/ref_stubs.o"
  g++ -shared -fopenmp -Wl,--no-undefined -o "$OUT/libleonard_ref_$name.so" "${objs[@]}" "$objdir/ref_harness.o" \
      "$objdir/ref_stubs.o"
}
COMMON=(-O2 -fPIC -fopenmp -std=c++17 -w -include ctime -include cstring -I"$HERE/eigen_shim" -I"$HERE/xdr_shim" -I"$REF"
        -DMBE="\"$REF/utils/MatrixBaseExtension.h\"" -DEIGEN -DMULTITHREADING)
build su3 "${COMMON[@]}" -DNUMCOLORS=3
build su2adj "${COMMON[@]}" -DNUMCOLORS=2 -DADJOINT
build su3_native "${COMMON[@]}" -march=native -DNUMCOLORS=3
gcc -march=native -Q --help=target 2>/dev/null | grep -E '^\s+-march=' | head -1 | awk '{print $2}' > "$OUT/native_arch.txt"
# the C++ adapter of include/ compiled against the reference's own headers, in a driver
# (oracle/adapter_driver.cpp) linked with the reference's objects and the GPU library
LIBDIR="$HERE/../leonardym_b200"
for name in su3 su2adj; do
  if [ "$name" = su3 ]; then flags=(-DNUMCOLORS=3); else flags=(-DNUMCOLORS=2 -DADJOINT); fi
  objdir="$OUT/obj_$name"
  g++ "${COMMON[@]}" "${flags[@]}" -I"$HERE/../include" -c "$HERE/adapter_driver.cpp" -o "$objdir/adapter_driver.o"
  if [ -f "$LIBDIR/liblym_b200.so" ]; then
    g++ -fopenmp -o "$OUT/adapter_driver_$name" "$objdir"/*.o -L"$LIBDIR" -llym_b200 \
        -Wl,-rpath,'$ORIGIN/../../leonardym_b200'
  fi
done
