#!/usr/bin/env bash
# Builds the reference's own CUDA time step (test infrastructure: the golden-
# vector generator and the reference arm of bench.py) from the unmodified
# sources in the reference checkout, one executable per grid configuration:
#
#     oracle/_ref/<cfg>/refdrv        the reference's solver.o + fftfuncs.o (cuFFT)
#     oracle/_ref/<cfg>/refdrv_gnss   the same program linked against the B200
#                                     library through gnss-1_b200/refabi/refabi.cu
#
# The reference fixes every size and parameter at compile time in dnsparams.h
# (dnsparams.h:9-41).  For each configuration this script creates
# oracle/_ref/<cfg>/src/ holding symbolic links to the reference's .cu/.h files
# plus a generated dnsparams.h; compiling the links from that directory makes
# the quoted include "dnsparams.h" resolve to the generated one.  Nothing from
# the reference is copied, and oracle/_ref/ is not committed.  The CUDA-samples
# headers the reference includes are replaced by oracle/refshim/.
#
# usage: oracle/build_ref.sh [cfg ...]      (default: all configurations)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${GNSS_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
LIB="$HERE/../gnss-1_b200"
FLAGS=(-O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -w -w)

if [ ! -f "$REF/solver.cu" ]; then
    echo "build_ref.sh: reference sources not found in $REF" >&2
    exit 1
fi

# name  N (or NXxNYxNZ)  Re  Sc  Sc_c  alpha  dt  pert_amp (noise of the initial jet, initialize.cu:615-641)
#       [alias_filter (default 2/3; 15/16 is the reference's 15/32 rule, dnsparams.h:91)] [L in units of pi (default 2)]
CONFIGS="
g12    12   200.0   0.7  1.0   0.0    2.0e-3  0.0
g16    16   200.0   0.7  1.0   0.0    2.0e-3  0.0
g16a   16   200.0   0.7  1.0   0.05   2.0e-3  0.0
i16    16   200.0   0.7  1.0   0.0    2.0e-3  0.05
i32    32   1000.0  0.7  1.0   0.0    1.0e-3  0.05
c64    64   1000.0  0.7  0.7   0.0    1.0e-3  0.0
c128   128  1000.0  0.7  0.7   0.0    1.0e-3  0.0
c256   256  3000.0  0.7  1.0   0.0    5.0e-4  0.0
c512   512  5000.0  0.7  0.7   0.0    2.5e-4  0.0
n64y32 64x32x64 800.0 0.7 1.0  0.0    1.0e-3  0.0
a64    64   800.0   0.7  1.0   0.0    1.0e-3  0.0     (15.0/16.0)
l64    64   800.0   0.7  1.0   0.0    1.0e-3  0.0     (2.0/3.0)  4.0
r96a   96   800.0   0.7  1.0   0.05   1.0e-3  0.0
m48    48x96x64 800.0 0.7 1.0  0.0    1.0e-3  0.0
f48    48   800.0   0.7  1.0   0.0    1.0e-3  0.0     (1.0)
"

want=("$@")
SRCS=(solver cudafuncs fftfuncs allocate initialize iofuncs statistics)

gen_params() {  # N-or-NXxNYxNZ Re Sc Sc_c alpha dt pert_amp [alias_filter] [L/pi]
    local nx ny nz
    local af=${8:-"(2.0/3.0)"} lpi=${9:-2.0}
    IFS=x read -r nx ny nz <<< "$1"
    ny=${ny:-$nx}
    nz=${nz:-$nx}
    cat <<EOF
/* generated by oracle/build_ref.sh: the temporal-jet configuration of the
 * reference (dnsparams.h:9-41) with runtime sizes fixed for this build */
#define TX 8
#define TY 8
#define TZ 8
#define NX $nx
#define NY $ny
#define NZ $nz
#define NZ2 (NZ/2 + 1)
#define NN (NX*NY*NZ)
#define PI (M_PI)
#define LX ($lpi*PI)
#define LY ($lpi*PI)
#define LZ ($lpi*PI)
#define DX (LX/NX)
#define n_checkpoint 1000000
#define n_vis 1000000
#define n_stats 1000000
#define dt $6
#define nt 1
#define H (1.0)
#define theta (0.05)
#define theta_s (0.05)
#define theta_c (0.05)
#define Re $2
#define nu (H/Re)
#define Sc $3
#define Sc_c $4
#define alpha $5
#define alias_filter $af
#define pert_amp $7
#define rootdir "./"
#define sim_name "refdrv/"
#define RAD 1
EOF
}

build_one() {
    local name=$1 n=$2 re=$3 sc=$4 scc=$5 al=$6 dtv=$7 pert=$8 af=${9:-} lpi=${10:-}
    local d="$OUT/$name"
    mkdir -p "$d/src" "$d/obj"
    for f in "$REF"/*.cu "$REF"/*.h; do
        b=$(basename "$f")
        [ "$b" = "dnsparams.h" ] && continue
        ln -sf "$f" "$d/src/$b"
    done
    gen_params "$n" "$re" "$sc" "$scc" "$al" "$dtv" "$pert" $af $lpi > "$d/src/dnsparams.h"
    local objs=()
    for s in "${SRCS[@]}"; do
        # the reference is C++03 code (Makefile:2); C99 "complex double" needs it
        "$NVCC" "${FLAGS[@]}" -std=c++03 -dc -I"$HERE/refshim" -o "$d/obj/$s.o" "$d/src/$s.cu"
        objs+=("$d/obj/$s.o")
    done
    "$NVCC" "${FLAGS[@]}" -dc -I"$HERE/refshim" -I"$d/src" -o "$d/obj/refdriver.o" "$HERE/refdriver.cu"
    "$NVCC" "${FLAGS[@]}" -o "$d/refdrv" "${objs[@]}" "$d/obj/refdriver.o" -lcufft
    # drop-in variant: the same driver and the reference's remaining objects, with
    # solver.o and fftfuncs.o replaced by the B200 library's reference-ABI shim
    if [ -f "$LIB/libgnss_b200.so" ]; then
        "$NVCC" "${FLAGS[@]}" -dc -I"$HERE/../include" -I"$d/src" -o "$d/obj/refabi.o" \
            "$HERE/../gnss-1_b200/refabi/refabi.cu"
        local keep=()
        for o in "${objs[@]}"; do
            case "$(basename "$o")" in solver.o|fftfuncs.o) ;; *) keep+=("$o") ;; esac
        done
        "$NVCC" "${FLAGS[@]}" -o "$d/refdrv_gnss" "${keep[@]}" "$d/obj/refabi.o" "$d/obj/refdriver.o" \
            -L"$LIB" -lgnss_b200 -lcufft -Xlinker -rpath -Xlinker '$ORIGIN/../../../gnss-1_b200'
    fi
    # keep only the executables: the links into the reference tree stay here
    rm -rf "$d/src" "$d/obj"
    echo "built $d/refdrv"
}

pids=()
while read -r name n re sc scc al dtv pert af lpi; do
    [ -z "${name:-}" ] && continue
    if [ ${#want[@]} -gt 0 ]; then
        keep=0
        for w in "${want[@]}"; do [ "$w" = "$name" ] && keep=1; done
        [ $keep -eq 0 ] && continue
    fi
    build_one "$name" "$n" "$re" "$sc" "$scc" "$al" "$dtv" "$pert" $af $lpi &
    pids+=($!)
done <<< "$CONFIGS"
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
exit $rc
