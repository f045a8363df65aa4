# Builds the reference program (aav-antonov/F2M) from its sources where they lie,
# as a checker: the binary F2M.solver.exe goes to oracle/_ref/ (git-ignored) and
# is run only by tests/golden/make_reference_runs.py to record golden outputs.
# The recipe follows the reference's own makefile (nvcc for graph_cuda.cu,
# g++ -std=c++11 for the host stage, nvcc to link RUN.cpp); the only additions
# are the Boost stand-in header (refshim/) and an explicit sm_100a target.
# the reference checkout: $(F2M_REFERENCE), else a sibling directory named
# "reference" next to this repository
REF ?= $(if $(F2M_REFERENCE),$(F2M_REFERENCE),$(abspath ../../reference))
OUT := _ref
NVCC ?= /usr/local/cuda/bin/nvcc
CXX := $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
ARCH := -gencode arch=compute_100a,code=sm_100a
HOST := node E_thread V_thread comb_thread Ax_b
OBJS := $(OUT)/graph_cuda.o $(HOST:%=$(OUT)/%.o)

all: $(OUT)/F2M.solver.exe

$(OUT):
	mkdir -p $(OUT)

$(OUT)/graph_cuda.o: $(REF)/graph_cuda.cu | $(OUT)
	$(NVCC) $(ARCH) -I refshim -c $(REF)/graph_cuda.cu -o $@

$(OUT)/%.o: $(REF)/%.cpp | $(OUT)
	$(CXX) -std=c++11 -g -c $< -o $@

$(OUT)/F2M.solver.exe: $(OBJS) $(REF)/RUN.cpp
	$(NVCC) $(ARCH) -I refshim -o $@ $(OBJS) $(REF)/RUN.cpp

clean:
	rm -rf $(OUT)
