# Builds the unmodified fip reference (headless, NO_VIS) from its own sources into oracle/_ref/.
# Test infrastructure only: the binaries are the parity pin for the CPU oracle and for the
# CUDA solver. Nothing here is shipped or linked into the product.
#
#   make -f oracle/ref.mk REF=<reference checkout>     (run from the repository root)
#
# Three binaries are produced, all from the reference's sources where they lie:
#   _ref/fip_ref         as shipped (wet/dry mask on, host reads the CFL slots unsynchronised)
#   _ref/fip_ref_nomask  src/kernels.cu with ENABLE_MASK 0 (patched copy under _ref/patched/; the
#                        store_mask() call also gets a literal 0, since the shipped file does not
#                        compile with the mask off: mask_new is only declared under ENABLE_MASK)
#   _ref/fip_ref_sync    nomask + a cudaDeviceSynchronize() at the top of controlTimestep(), so
#                        variable_dt reads the CFL slots of the step that just ran (deterministic)
# The patched copies are generated by sed at build time into _ref/patched/ (git-ignored); the
# reference's own build system (CMake) is not used.

REF      ?= $(FIP_REFERENCE_SRC)
ifeq ($(REF),)
$(error set REF=<reference checkout> or FIP_REFERENCE_SRC)
endif
OUT      := oracle/_ref
CUDA     ?= /usr/local/cuda
NVCC     := $(CUDA)/bin/nvcc
CXX      ?= g++
ARCH     := -gencode arch=compute_100a,code=sm_100a
YAML     := $(REF)/deps/yaml-cpp
INC      := -I$(REF)/src -I$(REF)/deps -I$(YAML)/include -I$(CUDA)/include
CXXFLAGS := -std=c++20 -O2 -DNO_VIS -w
NVFLAGS  := -std=c++17 -O3 $(ARCH) -use_fast_math -extended-lambda -DNO_VIS -w
LIBS     := -L$(CUDA)/lib64 -lnvrtc -lcuda -lcudart -ldl -lpthread

YAML_SRC := $(wildcard $(YAML)/src/*.cpp) $(wildcard $(YAML)/src/contrib/*.cpp)
YAML_OBJ := $(patsubst $(YAML)/src/%.cpp,$(OUT)/obj/yaml/%.o,$(YAML_SRC))
HOST_SRC := simdata boundary_condition timeseries bc_kernel_gen
HOST_OBJ := $(HOST_SRC:%=$(OUT)/obj/%.o)

all: $(OUT)/fip_ref $(OUT)/fip_ref_nomask $(OUT)/fip_ref_sync

$(OUT)/obj/yaml/%.o: $(YAML)/src/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -I$(YAML)/include -I$(YAML)/src -c $< -o $@

$(OUT)/obj/%.o: $(REF)/src/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) $(INC) -c $< -o $@

# --- as shipped -------------------------------------------------------------------------------
$(OUT)/obj/main.o: $(REF)/src/main.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) $(INC) -c $< -o $@

$(OUT)/obj/kernels.o: $(REF)/src/kernels.cu
	@mkdir -p $(dir $@)
	$(NVCC) $(NVFLAGS) $(INC) -c $< -o $@

$(OUT)/fip_ref: $(OUT)/obj/main.o $(OUT)/obj/kernels.o $(HOST_OBJ) $(YAML_OBJ)
	$(NVCC) $(ARCH) $^ -o $@ $(LIBS)

# --- mask off ---------------------------------------------------------------------------------
$(OUT)/patched/kernels_nomask.cu: $(REF)/src/kernels.cu oracle/ref.mk
	@mkdir -p $(dir $@)
	sed -e 's/^#define ENABLE_MASK 1/#define ENABLE_MASK 0/' \
	    -e 's/store_mask(mask, mask_new,/store_mask(mask, 0,/' $< > $@
	grep -q '^#define ENABLE_MASK 0' $@

$(OUT)/obj/kernels_nomask.o: $(OUT)/patched/kernels_nomask.cu
	$(NVCC) $(NVFLAGS) $(INC) -c $< -o $@

$(OUT)/fip_ref_nomask: $(OUT)/obj/main.o $(OUT)/obj/kernels_nomask.o $(HOST_OBJ) $(YAML_OBJ)
	$(NVCC) $(ARCH) $^ -o $@ $(LIBS)

# --- mask off + synchronised CFL readback -----------------------------------------------------
$(OUT)/patched/main_sync.cpp: $(REF)/src/main.cpp oracle/ref.mk
	@mkdir -p $(dir $@)
	sed 's/^void controlTimestep()$$/void controlTimestep_unsynced();\nvoid controlTimestep() { cudaDeviceSynchronize(); controlTimestep_unsynced(); }\nvoid controlTimestep_unsynced()/' $< > $@
	grep -q 'controlTimestep_unsynced' $@

$(OUT)/obj/main_sync.o: $(OUT)/patched/main_sync.cpp
	$(CXX) $(CXXFLAGS) $(INC) -c $< -o $@

$(OUT)/fip_ref_sync: $(OUT)/obj/main_sync.o $(OUT)/obj/kernels_nomask.o $(HOST_OBJ) $(YAML_OBJ)
	$(NVCC) $(ARCH) $^ -o $@ $(LIBS)

clean:
	rm -rf $(OUT)

.PHONY: all clean
