# Builds the reference's own program (opencfd.c and every object of src/,
# compiled by ref.mk from the sources where they lie) with its RHS-path
# calls served by libocfd_b200 through opencfd-scu_b200/glue/ocfd_b200_glue.cu.
# The six functions the glue provides (du_comput, OCFD_time_advance,
# get_duvwT, get_Amu, OCFD_bc, filtering) are renamed in the reference's
# objects that define them, so the driver's calls resolve to the glue; no
# reference source is edited or copied.
#   make -f oracle/dropin.mk REF_DIR=/root/reference      (after ref.mk)
# Output: oracle/_ref/dropin/opencfd-scu-dropin.out (git-ignored; travels to
# the GPU box with the library it loads from opencfd-scu_b200/).
# TEST INFRASTRUCTURE: it proves the drop-in boundary.
HERE    := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
ROOT    := $(abspath $(HERE)..)
REF_DIR ?= /root/reference
REFOBJ  := $(HERE)_ref/obj
OUT     := $(HERE)_ref/dropin
SHIM    := $(HERE)mpi_shim
LIBDIR  := $(ROOT)/opencfd-scu_b200
CUDA    ?= /usr/local/cuda
NVCC    := $(CUDA)/bin/nvcc
ARCH    := -gencode arch=compute_100a,code=sm_100a

# objects whose definitions of the six functions give way to the glue's
RENAME  := OCFD_Stream OCFD_time commen_kernel OCFD_boundary OCFD_filtering
SYMS    := --redefine-sym du_comput=ocfd_ref_du_comput \
           --redefine-sym OCFD_time_advance=ocfd_ref_OCFD_time_advance \
           --redefine-sym get_duvwT=ocfd_ref_get_duvwT \
           --redefine-sym get_Amu=ocfd_ref_get_Amu \
           --redefine-sym OCFD_bc=ocfd_ref_OCFD_bc \
           --redefine-sym filtering=ocfd_ref_filtering

ALLOBJ  := $(wildcard $(REFOBJ)/*.o)
KEEP    := $(filter-out $(addprefix $(REFOBJ)/,$(addsuffix .o,$(RENAME))),$(ALLOBJ))
RENAMED := $(addprefix $(OUT)/,$(addsuffix .o,$(RENAME)))

all: $(OUT)/opencfd-scu-dropin.out

$(OUT):
	mkdir -p $@

$(OUT)/%.o: $(REFOBJ)/%.o | $(OUT)
	objcopy $(SYMS) $< $@

$(OUT)/glue.o: $(LIBDIR)/glue/ocfd_b200_glue.cu $(ROOT)/include/ocfd_b200.h | $(OUT)
	$(NVCC) -c -O2 -std=c++17 $(ARCH) -I$(SHIM) -I$(REF_DIR)/head -I$(ROOT)/include -w $< -o $@

# the library is found next to the repository's own build, relative to the binary
$(OUT)/opencfd-scu-dropin.out: $(KEEP) $(RENAMED) $(OUT)/glue.o $(LIBDIR)/libocfd_b200.so
	$(NVCC) -O3 $(ARCH) -o $@ $(KEEP) $(RENAMED) $(OUT)/glue.o -L$(LIBDIR) -locfd_b200 \
	    -Xlinker -rpath,'$$ORIGIN/../../../opencfd-scu_b200' -lm -lpthread

clean:
	rm -rf $(OUT)

.PHONY: all clean
