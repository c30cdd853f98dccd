#!/usr/bin/env bash
# Builds the reference CPU_PIM solver, from the reference's own source file where it lies,
# into oracle/_ref/ (git-ignored).  TEST INFRASTRUCTURE ONLY: the outputs pin the oracle
# restatement and time the reference's CPU code; the solver never links them.
#
# No copy of the reference source is written anywhere: the source is streamed through
# sed (capacity constants only) into g++ together with ref_harness.cpp.
#
# Outputs:
#   _ref/libref_stock.so   capacity constants unchanged (MAXN 160, 10 replicas, 20 threads),
#                          Philox engine shim (ref_prelude.h)
#   _ref/libref_big.so     MAXN 256, 64 replicas, 64 threads, Philox engine shim
#   _ref/libref_big_mt.so  MAXN 256, 64 replicas, 256 threads, the reference's own
#                          std::mt19937 (no shim): the timed CPU baseline
#   _ref/cpu_pim_stock     the unmodified reference CLI (for output-format checks)
#   _ref/cpu_pim_philox    the reference CLI with stock capacities on the solver's Philox
#                          streams (ref_cli_main.cpp; for the CLI parity fixtures)
#   _ref/libref_tai.so     CPU-PIM/CPU_PIM_tai256c.cpp (n = 256, 92 active facilities hard-wired
#                          there; 10 replicas, 20 threads), Philox engine shim; its lumped draw
#                          goes to the shim's second engine (ref_prelude.h)
#
# The reference source path is $PIMQAP_REF_ROOT (default /root/reference).  When it is
# absent the script does nothing and exits 0.
set -euo pipefail

# PIMQAP_REF_ROOT names the reference checkout; unset, the conventional read-only mount of the
# build container is used, and the script says which source it builds from.
REF_ROOT="${PIMQAP_REF_ROOT:-/root/reference}"
[ -n "${PIMQAP_REF_ROOT:-}" ] || echo "build_ref.sh: PIMQAP_REF_ROOT unset, using $REF_ROOT"
SRC="$REF_ROOT/CPU-PIM/CPU_PIM.cpp"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
# The system g++ (libstdc++ linked dynamically, shared with the host process); $CXX may name
# a wrapper that links libstdc++ statically, which breaks iostream facets under Python.
CXX="${PIMQAP_REF_CXX:-/usr/bin/g++}"
# x86-64-v3 (AVX2/FMA/BMI2): runs on the GPU hosts as well as on the build container.
# Hidden visibility + -Bsymbolic: the reference's globals (N, I, D, F, beta, setup, ...) must
# bind inside the library, not to same-named symbols of the host process.
CXXFLAGS="-std=c++17 -O3 -march=x86-64-v3 -pthread -fPIC -w"
LIBFLAGS="-fvisibility=hidden -Wl,-Bsymbolic"

if [ ! -f "$SRC" ]; then
    echo "build_ref.sh: $SRC not found, reference harness not built"
    exit 0
fi
mkdir -p "$OUT"

# Exactly one line must match each capacity constant (and the last statement of main), or
# the recipe fails.
for pat in '^const int MAXN = 160;' '^const int MAXNUMREPLICAS = 10;' '^const int MAXNUMTHREADS = 20;' \
           '^    cout << "Elapsed time: " << duration.count() / 1000.0 << " seconds." << endl;$'; do
    c=$(grep -c "$pat" "$SRC" || true)
    if [ "$c" != "1" ]; then
        echo "build_ref.sh: pattern '$pat' matched $c lines in $SRC" >&2
        exit 1
    fi
done

# main() is renamed (ref_prelude.h), and a renamed int function that runs off its end is
# undefined behaviour (only main has the implicit return 0): the recipe adds that return 0
# after main's last statement.
patched() {  # maxn maxr maxt
    sed -e "s/^const int MAXN = 160;/const int MAXN = $1;/" \
        -e "s/^const int MAXNUMREPLICAS = 10;/const int MAXNUMREPLICAS = $2;/" \
        -e "s/^const int MAXNUMTHREADS = 20;/const int MAXNUMTHREADS = $3;/" \
        -e 's/^    cout << "Elapsed time: " << duration.count() \/ 1000.0 << " seconds." << endl;$/& return 0;/' "$SRC"
}

build_lib() {  # out maxn maxr maxt extra-flags
    local out="$1"; shift
    local maxn="$1" maxr="$2" maxt="$3"; shift 3
    { patched "$maxn" "$maxr" "$maxt"; cat "$HERE/ref_harness.cpp"; } |
        $CXX $CXXFLAGS $LIBFLAGS "$@" -shared -include "$HERE/ref_prelude.h" -x c++ - -o "$OUT/$out.tmp"
    mv "$OUT/$out.tmp" "$OUT/$out"
}

# CPU_PIM_tai256c.cpp: N becomes assignable (the harness loads instances), doMegaIteraTai
# takes the name the harness calls, and the lumped move's draw reads the shim's second engine.
TAI="$REF_ROOT/CPU-PIM/CPU_PIM_tai256c.cpp"
if [ -f "$TAI" ]; then
    for pat in '^const int N = 256;$' 'randomNonActiveIndex(rng\[t\])' \
               '^    cout << "Elapsed time: " << duration.count() / 1000.0 << " seconds." << endl;$'; do
        c=$(grep -c "$pat" "$TAI" || true)
        if [ "$c" != "1" ]; then
            echo "build_ref.sh: pattern '$pat' matched $c lines in $TAI" >&2
            exit 1
        fi
    done
    { sed -e 's/^const int N = 256;$/int N = 256;/' \
          -e 's/doMegaIteraTai/doMegaItera/g' \
          -e 's/randomNonActiveIndex(rng\[t\])/randomNonActiveIndex(pimqap_ref::lumped(rng[t]))/' \
          -e 's/^    cout << "Elapsed time: " << duration.count() \/ 1000.0 << " seconds." << endl;$/& return 0;/' "$TAI"
      cat "$HERE/ref_harness.cpp"; } |
        $CXX $CXXFLAGS $LIBFLAGS -shared -include "$HERE/ref_prelude.h" -x c++ - -o "$OUT/libref_tai.so.tmp"
    mv "$OUT/libref_tai.so.tmp" "$OUT/libref_tai.so"
fi

build_lib libref_stock.so 160 10 20
build_lib libref_big.so 256 64 64
build_lib libref_big_mt.so 256 64 256 -DPIMQAP_REF_NO_SHIM -mcmodel=medium
$CXX $CXXFLAGS "$SRC" -o "$OUT/cpu_pim_stock.tmp" && mv "$OUT/cpu_pim_stock.tmp" "$OUT/cpu_pim_stock"
{ patched 160 10 20; cat "$HERE/ref_harness.cpp"; } |
    $CXX $CXXFLAGS -include "$HERE/ref_prelude.h" -c -x c++ - -o "$OUT/cpu_pim_philox.o"
$CXX $CXXFLAGS "$HERE/ref_cli_main.cpp" "$OUT/cpu_pim_philox.o" -o "$OUT/cpu_pim_philox.tmp"
rm -f "$OUT/cpu_pim_philox.o"
mv "$OUT/cpu_pim_philox.tmp" "$OUT/cpu_pim_philox"
echo "build_ref.sh: built $(ls "$OUT" | tr '\n' ' ')"
