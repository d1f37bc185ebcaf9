# Builds the reference (RuanPetrus/cuda-graph-traversal) from its own
# sources, where they lie under REF_ROOT, into _ref/ (git-ignored).  Nothing
# is copied: nvcc reads REF_ROOT/src and REF_ROOT/examples directly.  MPI and
# NVSHMEM are replaced by the single-process shims in include/compat/shim
# (one rank, one PE: every NVSHMEM operation is a local load, store or
# atomic; a collective launch is a cooperative launch).
#
#   _ref/graph500_runner_ref  the reference's runner + library, unchanged
#   _ref/ref_dump             ref_dump.cu driving the reference library; dumps
#                             edges, CSR, BFS and SSSP outputs for fixtures
#   _ref/libref_host.so       ref_host.cu: the reference's host-side MRG code
#                             (jump table included) behind a C ABI
#   _ref/ref_bench            ref_bench.cu timing the reference library with
#                             its runner's protocol (selectable root counts)
# make -f ref.mk G5_REF_ROOT=<path to RuanPetrus/cuda-graph-traversal>
REF_ROOT ?= $(G5_REF_ROOT)
NVCC     ?= /usr/local/cuda/bin/nvcc
ARCH     ?= -gencode arch=compute_100a,code=sm_100a
SHIM     := ../include/compat/shim
FLAGS    := -O3 -Drestrict=__restrict__ -rdc=true $(ARCH) -I$(REF_ROOT)/src -I$(SHIM)
LIBSRC   := $(addprefix $(REF_ROOT)/src/,graph_generation.cu base.cu traversal.cu visualization.cu worker.cu)

all: _ref/graph500_runner_ref _ref/ref_dump _ref/libref_host.so _ref/ref_bench

_ref:
	mkdir -p _ref

_ref/graph500_runner_ref: $(LIBSRC) $(REF_ROOT)/examples/graph500_runner.cu | _ref
	$(NVCC) $(FLAGS) -o $@ $(LIBSRC) $(REF_ROOT)/examples/graph500_runner.cu -lm

_ref/ref_dump: ref_dump.cu $(LIBSRC) | _ref
	$(NVCC) $(FLAGS) -o $@ ref_dump.cu $(LIBSRC) -lm

_ref/ref_bench: ref_bench.cu $(LIBSRC) | _ref
	$(NVCC) $(FLAGS) -o $@ ref_bench.cu $(LIBSRC) -lm

_ref/libref_host.so: ref_host.cu | _ref
	$(NVCC) -O2 $(ARCH) -I$(REF_ROOT)/src -I$(SHIM) -Xcompiler -fPIC -shared -o $@ ref_host.cu

.PHONY: all
