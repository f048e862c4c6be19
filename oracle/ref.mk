# Builds the reference's own CPU LAPACK/BLAS path (lapack/*.c over blas/*.c) from
# its sources where they lie, into oracle/_ref/libref.so.  Test infrastructure only:
# the library is the checker and the CPU baseline, never part of the product.
#
#   make -f oracle/ref.mk REF=<reference tree>
#   (or CUCHOLESKY_REFERENCE=<reference tree> make -f oracle/ref.mk)
#
# The reference sources are not copied into this repository.  Three generated shims
# (written under oracle/_ref/shim/ only) let them compile on the CPU without a GPU:
#   * error.h / error.c : the reference's error.h and multigpu/error.c with its
#     cuGetErrorString renamed, because CUDA 12's cuda.h declares a different
#     cuGetErrorString(CUresult, const char **) (reference include/error.h:30).
#   * config.h          : stand-in for the header that blas/config.c generates on a
#     GPU at build time (blas/Makefile:50-57); the CPU routines never read it.
#   * <name>.fatbin.c   : empty device images; the CPU routines never load them.
# CUDA driver entry points referenced by the GPU halves of the same translation
# units resolve to oracle/ref_cuda_stub.c and are never called on the CPU path.
#
# No -ffast-math (reference lapack/Makefile:9 uses it): isnan() must survive so the
# info return on NaN inputs matches the source semantics.
REF   ?= $(CUCHOLESKY_REFERENCE)
ifeq ($(strip $(REF)),)
$(error set REF or CUCHOLESKY_REFERENCE to the reference source tree)
endif
HERE  := $(dir $(lastword $(MAKEFILE_LIST)))
OUT   := $(HERE)_ref
SHIM  := $(OUT)/shim
REFCC ?= gcc
CFLAGS_REF := -O2 -std=gnu99 -fopenmp -fPIC -march=x86-64-v3 -w

BLAS_SRC   := handle xerbla sgemm ssyrk strmm strsm cgemm cherk ctrmm ctrsm \
              dgemm dsyrk dtrmm dtrsm zgemm zherk ztrmm ztrsm
LAPACK_SRC := handle slauum spotrf spotri strtri dlauum dpotrf dpotri dtrtri \
              clauum cpotrf cpotri ctrtri zlauum zpotrf zpotri ztrtri \
              slogdet dlogdet clogdet zlogdet
FATBINS    := $(filter-out handle xerbla,$(BLAS_SRC) $(LAPACK_SRC))

OBJS := $(addprefix $(OUT)/obj/blas_,$(addsuffix .o,$(BLAS_SRC))) \
        $(addprefix $(OUT)/obj/lapack_,$(addsuffix .o,$(LAPACK_SRC))) \
        $(OUT)/obj/multigpu.o $(OUT)/obj/error.o $(OUT)/obj/stub.o

all: $(OUT)/libref.so

$(SHIM)/.stamp: $(HERE)ref.mk
	mkdir -p $(SHIM) $(OUT)/obj
	sed 's/cuGetErrorString/refGetErrorString/g' $(REF)/include/error.h > $(SHIM)/error.h
	sed 's/cuGetErrorString/refGetErrorString/g' $(REF)/multigpu/error.c > $(SHIM)/error.c
	printf '#ifndef CONFIG_H\n#define CONFIG_H\n' > $(SHIM)/config.h
	for p in S D C Z; do for v in N T C CN CC; do for d in MB NB KB; do \
	  printf '#define %sGEMM_%s_%s 64\n' $$p $$v $$d >> $(SHIM)/config.h; done; done; done
	printf '#define BANDWIDTH_HTOD 1.0\n#define BANDWIDTH_DTOH 1.0\n#define OVERHEAD_HTOD 1.0\n#define OVERHEAD_DTOH 1.0\n#endif\n' >> $(SHIM)/config.h
	for f in $(FATBINS); do printf 'static const unsigned char imageBytes[] = {0};\n' > $(SHIM)/$$f.fatbin.c; done
	touch $@

INC := -I$(SHIM) -I$(REF)/include -I/usr/local/cuda/include

$(OUT)/obj/blas_%.o: $(REF)/blas/%.c $(SHIM)/.stamp
	$(REFCC) $(CFLAGS_REF) $(INC) -I$(REF)/blas -c $< -o $@
$(OUT)/obj/lapack_%.o: $(REF)/lapack/%.c $(SHIM)/.stamp
	$(REFCC) $(CFLAGS_REF) $(INC) -I$(REF)/lapack -c $< -o $@
$(OUT)/obj/multigpu.o: $(REF)/multigpu/multigpu.c $(SHIM)/.stamp
	$(REFCC) $(CFLAGS_REF) $(INC) -c $< -o $@
$(OUT)/obj/error.o: $(SHIM)/.stamp
	$(REFCC) $(CFLAGS_REF) $(INC) -c $(SHIM)/error.c -o $@
$(OUT)/obj/stub.o: $(HERE)ref_cuda_stub.c $(SHIM)/.stamp
	$(REFCC) $(CFLAGS_REF) -I/usr/local/cuda/include -c $< -o $@

$(OUT)/libref.so: $(OBJS)
	$(REFCC) -shared -fopenmp -o $@ $(OBJS) -lm -lpthread

.PHONY: all
