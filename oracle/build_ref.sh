#!/usr/bin/env bash
# Compiles the reference ICON-GPU v1.2.9 from its sources, unmodified, for
# sm_100a into oracle/_ref/ (git-ignored; it travels to the GPU box with the
# rest of the working tree).  Test infrastructure only: the binaries are the
# reference that the oracle and the CUDA path are checked against.
#
#   oracle/_ref/ICON-GPU     the reference command-line tool
#   oracle/_ref/ref_harness  oracle/ref_harness.cu linked against the
#                            reference's cunfft_* / Iteration3 routines
#   oracle/_ref/ICONPreProcess  the stack pre-processing tool (plain C, gcc)
#   oracle/_ref/ICONMask3       the volume assembly / cross-validation mask
#                               tool (CUDA, cuFFT)
#
# The reference's own install script (IG/install) is not run: it calls nvcc
# without an architecture and links a prebuilt log object.  This recipe calls
# nvcc per source file with -gencode for sm_100a and replaces the log object
# with oracle/ref_logstub.c.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${ICON_REFERENCE_ROOT:-/root/reference}"
SRC="$REF_ROOT/tomography/ICON_GPU_v1.2.9/sourceCode/ICON-GPU"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -d "$SRC" ]; then
    echo "build_ref: reference sources not found at $SRC; skipping" >&2
    exit 0
fi
mkdir -p "$OBJ"
ARCH="-gencode arch=compute_100a,code=sm_100a"
NVCC="${NVCC:-nvcc}"
CU="ICONGPU readSlicePart readSlicePart_crossV MainCode MainCode_crossV nufft_gpu_v8 Iteration2 alpha_new2 saveMRC saveMRC_real px2D weight reProject_NFFT calFRC"
for f in $CU; do
    if [ ! -f "$OBJ/$f.o" ] || [ "$SRC/$f.cu" -nt "$OBJ/$f.o" ]; then
        "$NVCC" $ARCH -w -I"$SRC" -o "$OBJ/$f.o" -c "$SRC/$f.cu"
    fi
done
gcc -w -O2 -c "$SRC/mrcfile3.c" -o "$OBJ/mrcfile3.o"
gcc -O2 -c "$HERE/ref_logstub.c" -o "$OBJ/ref_logstub.o"
LIBS="$OBJ/readSlicePart_crossV.o $OBJ/MainCode_crossV.o $OBJ/readSlicePart.o $OBJ/MainCode.o $OBJ/nufft_gpu_v8.o $OBJ/Iteration2.o $OBJ/saveMRC_real.o $OBJ/alpha_new2.o $OBJ/mrcfile3.o $OBJ/saveMRC.o $OBJ/px2D.o $OBJ/weight.o $OBJ/reProject_NFFT.o $OBJ/calFRC.o $OBJ/ref_logstub.o"
"$NVCC" $ARCH -o "$OUT/ICON-GPU" "$OBJ/ICONGPU.o" $LIBS -lcufft -lpthread
"$NVCC" $ARCH -w -I"$SRC" -o "$OUT/ref_harness" "$HERE/ref_harness.cu" $LIBS -lcufft -lpthread
SC="$REF_ROOT/tomography/ICON_GPU_v1.2.9/sourceCode"
PP="$SC/ICONPreProcess"
gcc -w -O2 -o "$OUT/ICONPreProcess" "$PP/ICONPreProcess.c" "$PP/mrcfile3.c" "$HERE/ref_logstub.c" -lm
MK="$SC/ICONMask3"
"$NVCC" $ARCH -w -I"$MK" -o "$OBJ/ICONMask3.o" -c "$MK/ICONCrossVMaskIn2D_weightOnlyOnSampled.cu"
gcc -w -O2 -c "$MK/mrcfile3.c" -o "$OBJ/mk_mrcfile3.o"
"$NVCC" $ARCH -o "$OUT/ICONMask3" "$OBJ/ICONMask3.o" "$OBJ/mk_mrcfile3.o" "$OBJ/ref_logstub.o" -lcufft
echo "build_ref: built $OUT/ICON-GPU, $OUT/ref_harness, $OUT/ICONPreProcess and $OUT/ICONMask3"
