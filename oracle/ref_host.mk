# CHECKER ONLY: builds two host stages of the reference's own main.cpp and
# HPM.cpp (HPM-MVS++, read in place from $(REF)) for the CPU:
# ConfidenceEvaluation and RunFusion / RunFusion_Sky_Strict, exported by
# ref_host_driver.cpp, into oracle/_ref/libhpmref_host.so.  OpenCV is replaced
# by ref_shim_host/cv_host.hpp; unreachable code (the CUDA and OpenCV calls of
# the other stages) is dropped by -ffunction-sections / --gc-sections, and the
# link refuses any symbol left undefined.  No reference source is copied.
# Flags: the reference's README builds with a plain `cmake ..` (no build type),
# so its host code gets no optimisation flags and no -ffast-math
# (CMakeLists.txt:11-19); -O2 changes no IEEE result on x86-64 (no FMA
# contraction without -mfma).  OpenMP is left off so that ExportPointCloud's
# parallel loop (HPM.cpp:464) writes the points in order.
#   make -f ref_host.mk REF=<reference source tree>
# REF: the reference's source tree (HPM.cu, HPM.h, main.h, main.cpp, HPM.cpp); no default
ifndef REF
$(error set REF to the reference's source tree: make -f ref_host.mk REF=<reference source tree>)
endif
HOSTCC := $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
OUT := _ref
FLAGS := -std=c++14 -O2 -fPIC -ffunction-sections -fdata-sections -fvisibility=hidden -w \
         -I ref_shim_host -I $(REF) -I /usr/local/cuda/include
SHIM := ref_shim_host/cv_host.hpp

all: $(OUT)/libhpmref_host.so

$(OUT)/host_main.o: $(REF)/main.cpp $(REF)/main.h $(REF)/HPM.h $(SHIM)
	@mkdir -p $(OUT)
	$(HOSTCC) $(FLAGS) -Dmain=hpm_reference_main_unused -c $< -o $@

$(OUT)/host_HPM.o: $(REF)/HPM.cpp $(REF)/main.h $(REF)/HPM.h $(SHIM)
	@mkdir -p $(OUT)
	$(HOSTCC) $(FLAGS) -c $< -o $@

$(OUT)/host_driver.o: ref_host_driver.cpp $(REF)/main.h $(REF)/HPM.h $(SHIM)
	@mkdir -p $(OUT)
	$(HOSTCC) $(FLAGS) -c $< -o $@

$(OUT)/libhpmref_host.so: $(OUT)/host_main.o $(OUT)/host_HPM.o $(OUT)/host_driver.o
	$(HOSTCC) -shared -Wl,--gc-sections -Wl,--no-undefined -o $@ $^

.PHONY: all
