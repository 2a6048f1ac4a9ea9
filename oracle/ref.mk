# Builds the reference (OpenCFD-SCU) as a checker: its own sources, compiled
# where they lie, for sm_100a, linked against the single-rank MPI shim.
# Outputs go to oracle/_ref/ only (git-ignored; travels to the GPU box).
#   make -f oracle/ref.mk REF_DIR=/root/reference
# TEST INFRASTRUCTURE ONLY.  No source of the reference is copied.
HERE    := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
REF_DIR ?= /root/reference
OUT     := $(HERE)_ref
SHIM    := $(HERE)mpi_shim
CUDA    ?= /usr/local/cuda
NVCC    := $(CUDA)/bin/nvcc
HOSTCC  := $(if $(wildcard /usr/bin/gcc),/usr/bin/gcc,gcc)

CU_SRC  := $(wildcard $(REF_DIR)/src/*.cu)
C_SRC   := $(wildcard $(REF_DIR)/src/*.c)
CU_OBJ  := $(patsubst $(REF_DIR)/src/%.cu,$(OUT)/obj/%.o,$(CU_SRC))
C_OBJ   := $(patsubst $(REF_DIR)/src/%.c,$(OUT)/obj/%.o,$(C_SRC))

# same optimisation level as the reference makefile (-O3), target sm_100a
NVFLAGS := -dc -O3 -gencode arch=compute_100a,code=sm_100a -I$(SHIM) -I$(REF_DIR)/head -w
CFLAGS  := -c -std=gnu99 -O3 -I$(SHIM) -I$(REF_DIR)/head -I$(CUDA)/include -w

all: $(OUT)/opencfd-scu.out

$(OUT)/obj:
	mkdir -p $@

$(OUT)/obj/%.o: $(REF_DIR)/src/%.cu | $(OUT)/obj
	$(NVCC) $(NVFLAGS) $< -o $@

$(OUT)/obj/%.o: $(REF_DIR)/src/%.c | $(OUT)/obj
	$(HOSTCC) $(CFLAGS) $< -o $@

$(OUT)/obj/opencfd.o: $(REF_DIR)/opencfd.c | $(OUT)/obj
	$(HOSTCC) $(CFLAGS) $< -o $@

$(OUT)/obj/mpi_shim.o: $(SHIM)/mpi_shim.c $(SHIM)/mpi.h | $(OUT)/obj
	$(HOSTCC) -c -O2 -std=gnu99 -I$(SHIM) $< -o $@

$(OUT)/opencfd-scu.out: $(OUT)/obj/opencfd.o $(CU_OBJ) $(C_OBJ) $(OUT)/obj/mpi_shim.o
	$(NVCC) -O3 -gencode arch=compute_100a,code=sm_100a -o $@ $^ -lm -lpthread

clean:
	rm -rf $(OUT)

.PHONY: all clean
