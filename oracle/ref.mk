# Recipe that compiles the REFERENCE's own CUDA sources (RapidsAtHKUST/cuGridder,
# read where they lie under REF) for sm_100a into oracle/_ref/libcurafft_ref.so.
#
# Test infrastructure only: the library is a parity checker.  It is run on a
# B200 by tests/golden/make_golden.py to record golden outputs, and by the
# reference-CUDA timing of bench.py --impl reference when present.  Nothing is
# copied from the reference tree; objects and the .so go to oracle/_ref/
# (git-ignored, travels to the GPU box with the snapshot).
#
#   make -f oracle/ref.mk -j8          (from the repo root)
#
# It also builds oracle/_ref/libref_bins.so from oracle/ref_bins.cu (test code
# of this repository) against that library: the reference's binning stage
# with its hive offsets and per-cell counts read back.
#
# Flags follow the reference's own build line (Makefile:15-16): -O3,
# --default-stream per-thread, -use_fast_math, relocatable device code, FP64
# objects plus FP32 objects built with -DSINGLE.  -lnvToolsExt is dropped
# (absent in CUDA 12.9, no NVTX call exists in the sources).
REF ?= /root/reference
OUT := oracle/_ref
NVCC ?= nvcc
HOSTCXX := $(firstword $(wildcard /usr/bin/g++) g++)
HOSTCC := $(firstword $(wildcard /usr/bin/gcc) gcc)
NVFLAGS := -std=c++14 -ccbin=$(HOSTCXX) -O3 -gencode arch=compute_100a,code=sm_100a \
           -Wno-deprecated-gpu-targets --default-stream per-thread \
           -Xcompiler "-fPIC -O3" -use_fast_math -lineinfo -w
INC := -I$(REF)/include -I$(REF)/include/cuda_sample -I$(REF)/contrib

SRC_COMMON_CU := src/common_utils.cu
SRC_COMMON_C := contrib/legendre_rule_fast.c
SRC_PREC := src/fourier/conv_interp_invoker.cu src/fourier/conv.cu src/fourier/interp.cu \
            src/fourier/cuft.cu src/fourier/deconv.cu src/astro/cugridder.cu \
            src/astro/precomp.cu src/astro/ra_exec.cu src/utils.cu \
            contrib/common.cu contrib/utils_fp.cu

flat = $(subst /,_,$(basename $(1)))
OBJ_COMMON := $(OUT)/obj/$(call flat,$(SRC_COMMON_CU)).o $(OUT)/obj/$(call flat,$(SRC_COMMON_C)).o
OBJ_64 := $(foreach s,$(SRC_PREC),$(OUT)/obj/$(call flat,$(s)).o)
OBJ_32 := $(foreach s,$(SRC_PREC),$(OUT)/obj/$(call flat,$(s))_32.o)

all: $(OUT)/libcurafft_ref.so $(OUT)/libref_bins.so

$(OUT)/obj:
	mkdir -p $@

define cu64
$(OUT)/obj/$(call flat,$(1)).o: $(REF)/$(1) | $(OUT)/obj
	$(NVCC) --device-c -c $(NVFLAGS) $(INC) $$< -o $$@
endef
define cu32
$(OUT)/obj/$(call flat,$(1))_32.o: $(REF)/$(1) | $(OUT)/obj
	$(NVCC) -DSINGLE --device-c -c $(NVFLAGS) $(INC) $$< -o $$@
endef
$(foreach s,$(SRC_PREC) $(SRC_COMMON_CU),$(eval $(call cu64,$(s))))
$(foreach s,$(SRC_PREC),$(eval $(call cu32,$(s))))

$(OUT)/obj/$(call flat,$(SRC_COMMON_C)).o: $(REF)/$(SRC_COMMON_C) | $(OUT)/obj
	$(HOSTCC) -c -fPIC -O3 $(INC) $< -o $@

$(OUT)/libcurafft_ref.so: $(OBJ_COMMON) $(OBJ_64) $(OBJ_32)
	$(NVCC) -shared $(NVFLAGS) $^ -o $@ -lm -lcudart -lcufft

# the binning harness (oracle/ref_bins.cu, this repository's test code) calls
# the FP64 reference functions of libcurafft_ref.so through their own headers
$(OUT)/libref_bins.so: oracle/ref_bins.cu $(OUT)/libcurafft_ref.so
	$(NVCC) -shared $(NVFLAGS) $(INC) $< -o $@ -L$(OUT) -lcurafft_ref -lcudart \
	    -Xlinker -rpath,'$$ORIGIN'

clean:
	rm -rf $(OUT)

.PHONY: all clean
