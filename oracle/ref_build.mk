# CHECKER ONLY: builds the reference's own CUDA code (HPM.cu of HPM-MVS++, read
# in place from $(REF)) for sm_100a with the reference's nvcc flags
# (CMakeLists.txt:10, arch changed from sm_86), plus ref_driver.cu, into
# oracle/_ref/libhpmref.so.  OpenCV is replaced by type stand-ins
# (ref_shim/opencv2) and curand seeding by ref_shim/ref_rng.h; no reference
# source is copied.   make -f ref_build.mk REF=<reference source tree>
# REF: the reference's source tree (HPM.cu, HPM.h, main.h, main.cpp, HPM.cpp); no default
ifndef REF
$(error set REF to the reference's source tree: make -f ref_build.mk REF=<reference source tree>)
endif
NVCC ?= /usr/local/cuda/bin/nvcc
HOSTCC := $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
OUT := _ref
FLAGS := -O3 --use_fast_math --maxrregcount=128 -std=c++14 -gencode arch=compute_100a,code=sm_100a \
         -ccbin $(HOSTCC) -Xcompiler -fPIC -w -I ref_shim -I $(REF) -I ../include

all: $(OUT)/libhpmref.so

$(OUT)/HPM.o: $(REF)/HPM.cu $(REF)/HPM.h $(REF)/main.h ref_shim/ref_rng.h ref_shim/cv_stub.hpp
	@mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -rdc=true -include ref_shim/ref_rng.h -c $(REF)/HPM.cu -o $@

$(OUT)/ref_driver.o: ref_driver.cu $(REF)/HPM.h ref_shim/cv_stub.hpp
	@mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -rdc=true -c ref_driver.cu -o $@

$(OUT)/libhpmref.so: $(OUT)/HPM.o $(OUT)/ref_driver.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -ccbin $(HOSTCC) -shared -o $@ $^ -cudart static

.PHONY: all
