# ORACLE (test infrastructure): builds the reference from its own sources in
# /root/reference (never copied into this repository) for sm_100a. Outputs go
# only to _ref/ (git-ignored, shipped to the GPU box with the tree).
#   make -C oracle -f ref.mk
# Differences from the upstream Makefile (which builds for sm_35 with -G):
#   - -O2 device code (no -G); the warp intrinsics are mapped by ref/shim.h;
#   - io/IO.cpp is compiled as C++03 (it returns `false` from a Graph*
#     function, io/IO.cpp:137-138, which C++11 rejects);
#   - main/run.cpp is compiled as CUDA (it includes match/Match.h);
#   - readline headers are empty stubs (util/Util.h includes them, nothing
#     calls them).
REF ?= /root/reference
OUT := _ref
NVCC ?= /usr/local/cuda/bin/nvcc
ARCH := -gencode arch=compute_100a,code=sm_100a
SHIM := -include ref/shim.h -Iref/stub
OBJS := $(OUT)/Util.o $(OUT)/Graph.o $(OUT)/IO.o $(OUT)/Match.o

all: $(OUT)/GpSM.exe $(OUT)/ref_driver $(OUT)/run_dropin

# The reference's own driver main/run.cpp, unmodified, compiled against this
# library's drop-in Graph/IO/Match (include/gpsm_host/) and linked with
# libgpsm.so. It is fed to the compiler on standard input from
# ref/dropin/main/, so its `#include "../io/IO.h"` lines resolve to the shim
# headers under ref/dropin/ instead of the reference's own classes.
LIBDIR := $(abspath ../gpsm_b200)
$(OUT)/run_dropin: $(REF)/main/run.cpp $(wildcard ref/dropin/*/*.h) $(LIBDIR)/libgpsm.so | $(OUT)
	cd ref/dropin/main && g++ -O2 -w -std=c++17 -I$(abspath ../include) -x c++ - -o $(abspath $@) \
	  -L$(LIBDIR) -lgpsm -Wl,-rpath,'$$ORIGIN/../../gpsm_b200' < $(REF)/main/run.cpp

$(OUT):
	mkdir -p $(OUT)

$(OUT)/Util.o: $(REF)/util/Util.cpp | $(OUT)
	g++ -O2 -w -Iref/stub -c $< -o $@
$(OUT)/Graph.o: $(REF)/graph/Graph.cpp | $(OUT)
	g++ -O2 -w -Iref/stub -c $< -o $@
$(OUT)/IO.o: $(REF)/io/IO.cpp | $(OUT)
	g++ -O2 -w -std=c++03 -Iref/stub -c $< -o $@
$(OUT)/Match.o: $(REF)/match/Match.cu ref/shim.h | $(OUT)
	$(NVCC) $(ARCH) -O2 -w $(SHIM) -c $< -o $@
$(OUT)/run.o: $(REF)/main/run.cpp ref/shim.h | $(OUT)
	$(NVCC) $(ARCH) -O2 -w $(SHIM) -x cu -c $< -o $@
$(OUT)/ref_driver.o: ref/ref_driver.cpp ref/shim.h | $(OUT)
	$(NVCC) $(ARCH) -O2 -w $(SHIM) -I$(REF) -x cu -c $< -o $@
$(OUT)/GpSM.exe: $(OUT)/run.o $(OBJS)
	$(NVCC) $(ARCH) $^ -o $@
$(OUT)/ref_driver: $(OUT)/ref_driver.o $(OBJS)
	$(NVCC) $(ARCH) $^ -o $@

clean:
	rm -rf $(OUT)
.PHONY: all clean
