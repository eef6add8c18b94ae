# Builds the reference's accuracy drivers UNCHANGED, from their sources where
# they lie under the reference tree, against this project's compat libraries
# (mcfft_b200/libmcfft_{1,2,3}d.so) and the FFTW-named oracle shim.  Test
# infrastructure: outputs go to oracle/_ref/ (git-ignored; travels to the GPU
# box).  Only builds where the reference is mounted.
#   make -C oracle -f drivers.mk
# The reference tree: MCFFT_REF_DIR, else the directory beside the repository.
MCFFT_REF_DIR ?= $(abspath ../../reference)
REF := $(MCFFT_REF_DIR)
OUT := _ref
CXX_ := /usr/bin/g++
CC_ := /usr/bin/gcc
MC := ../mcfft_b200
FLAGS := -O2 -w -fopenmp

CUDA_LIB := /usr/local/cuda/lib64

all: $(OUT)/accuracy_1d $(OUT)/accuracy_2d $(OUT)/accuracy_3d $(OUT)/handle_caller_1d \
     $(OUT)/handle_caller_2d

$(OUT)/shim.o: fftw_compat/fftw_shim.c fftw_compat/fftw3.h
	mkdir -p $(OUT)
	$(CC_) $(FLAGS) -Ifftw_compat -c $< -o $@

$(OUT)/fft64.o: fft64.c
	mkdir -p $(OUT)
	$(CC_) $(FLAGS) -fPIC -c $< -o $@

$(OUT)/accuracy_%d: $(REF)/benchmark/accuracy_%d.cpp $(OUT)/shim.o $(OUT)/fft64.o $(MC)/libmcfft_%d.so
	$(CXX_) $(FLAGS) -std=c++14 -Ihip_stub -Ifftw_compat $< $(OUT)/shim.o $(OUT)/fft64.o \
	  -L$(MC) -lmcfft_$*d -Wl,-rpath,'$$ORIGIN/../../mcfft_b200' -o $@

# handle_caller.cpp (this directory) against the reference's own
# include/mcfft_{1,2}d_device.h: its handle struct, passed by value.
$(OUT)/handle_caller_%d: handle_caller.cpp $(REF)/include/mcfft_%d_device.h $(OUT)/fft64.o $(MC)/libmcfft_%d.so
	$(CXX_) $(FLAGS) -std=c++14 -DCALLER_DIM=$* -Ihip_stub -I$(REF)/include $< $(OUT)/fft64.o \
	  -L$(MC) -lmcfft_$*d -L$(CUDA_LIB) -lcudart \
	  -Wl,-rpath,'$$ORIGIN/../../mcfft_b200' -Wl,-rpath,$(CUDA_LIB) -o $@

clean:
	rm -rf $(OUT)

.PHONY: all clean
