# Compiles the reference's own CUDA sources (GPUcomcot.cu, GPUMass_s.cu,
# GPUMoment_s.cu, GPUOpen_BD.cu, GPUall_grids.cu, GPUOutput.cu) where they lie,
# for sm_100a, into oracle/_ref/.  Used only to generate the golden vectors that
# pin the CPU oracle (oracle/make_ref_goldens.py); never part of the product.
# Two builds: the reference's own flags (nvcc default FMA contraction, as its
# Makefile:13 builds it) and one with -fmad=false, whose float rounding follows
# the source order exactly.
# The reference checkout: COMCOT_REFERENCE_DIR, else the default below.  When
# its sources are absent (a machine without the reference) nothing is built
# and the prebuilt oracle/_ref libraries, if any, are used as they are.
REF     ?= $(or $(COMCOT_REFERENCE_DIR),/root/reference)
NVCC    ?= nvcc
SRCS    := GPUcomcot.cu GPUMass_s.cu GPUMoment_s.cu GPUOpen_BD.cu GPUall_grids.cu GPUOutput.cu
ARCH    := -gencode arch=compute_100a,code=sm_100a
OUT     := _ref

ifeq ($(wildcard $(REF)/GPUMass_s.cu),)
all:
	@echo "ref.mk: no reference sources at $(REF); skipping"
else
all: $(OUT)/libref_gpu.so $(OUT)/libref_gpu_nofma.so
endif

$(OUT)/libref_gpu.so: $(addprefix $(REF)/,$(SRCS))
	@mkdir -p $(OUT)
	$(NVCC) $(ARCH) -O3 -rdc=true -Xcompiler -fPIC -shared -I$(REF) -w -o $@ $(addprefix $(REF)/,$(SRCS))

$(OUT)/libref_gpu_nofma.so: $(addprefix $(REF)/,$(SRCS))
	@mkdir -p $(OUT)
	$(NVCC) $(ARCH) -O3 -fmad=false -rdc=true -Xcompiler -fPIC -shared -I$(REF) -w -o $@ $(addprefix $(REF)/,$(SRCS))

.PHONY: all
