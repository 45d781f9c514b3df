# Builds qcu itself (the reference library) from its own sources, for parity
# checks only.  Reads the read-only reference tree, writes nothing but
# oracle/_ref/.  Uses oracle/ref_stub/mpi.h in place of an MPI install; links
# the system NCCL, cuBLAS and cuRAND that qcu needs (CMakeLists.txt:19-23).
# The product never loads the result.
HERE    := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
# qcu's source tree: $(QCU_REFERENCE), else reference/ beside this repository
REF     ?= $(if $(QCU_REFERENCE),$(QCU_REFERENCE),$(abspath $(HERE)../../reference))
OUT     := $(HERE)_ref
NVCC    ?= nvcc
SRCS    := draft wilson_dslash clover_dslash lattice_cuda bistabcg \
           nccl_wilson_dslash nccl_wilson_bistabcg nccl_clover_dslash
# ref_timer.o is this project's harness that times qcu's wilson_dslash kernel
# with CUDA events; it is linked into the same library so that its launches
# and qcu's share one CUDA runtime
OBJS    := $(addprefix $(OUT)/,$(addsuffix .o,$(SRCS))) $(OUT)/ref_timer.o
FLAGS   := -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC \
           -I$(HERE)ref_stub -I$(REF)/include -w

all: $(OUT)/libqcu_ref.so

$(OUT)/%.o: $(REF)/src/%.cu
	@mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/ref_timer.o: $(HERE)ref_timer.cu
	@mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/libqcu_ref.so: $(OBJS)
	$(NVCC) -shared -gencode arch=compute_100a,code=sm_100a -o $@ $(OBJS) -lnccl -lcublas -lcurand

.PHONY: all

