# Builds the reference-derived checkers in oracle/_ref from the reference's own
# sources, where they lie (never copied into this repository).  Test
# infrastructure only; nothing here is linked into libgalpha.so.  The
# reference's cmake/GL build is not used.
#
#   _ref/libref.so       (g++)  host orient2d / incircle (gpudt/predicates.cpp)
#                               and the alpha predicates of
#                               gpudt/AlphaShape/predicates.h, host-compiled:
#                               birth times, attached test, exact comparisons
#   _ref/librefalpha.so  (nvcc) the reference's GPU alpha-shape engine,
#                               unmodified: gpudt/AlphaShape/Alpha_Shapes_2D.cu,
#                               kernel.cu, headers.cu for sm_100a, driven by
#                               ref_alpha_gpu.cu (Alpha_Shapes_2D(pInput, pDT)
#                               + computeAlphaShapes(), as main.cu:392-395)
#
# REF is the reference tree; the default is where this build keeps it and can
# be overridden (make -f ref.mk REF=/path/to/gAlpha2D).
REF ?= /root/reference
CXX ?= g++
NVCC ?= nvcc
FLAGS = -O2 -fPIC -ffp-contract=off -fno-fast-math -w
NVFLAGS = -gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -Xcompiler -fPIC -w
OUT = _ref
ALPHA = $(REF)/gpudt/AlphaShape

all: $(OUT)/libref.so $(OUT)/librefalpha.so

$(OUT)/libref.so: ref_pred.cpp ref_alpha.cpp
	mkdir -p $(OUT)
	$(CXX) $(FLAGS) -I$(REF)/gpudt -c $(REF)/gpudt/predicates.cpp -o $(OUT)/predicates.o
	$(CXX) $(FLAGS) -I$(REF)/gpudt -c ref_pred.cpp -o $(OUT)/ref_pred.o
	$(CXX) $(FLAGS) -I$(REF)/gpudt -c ref_alpha.cpp -o $(OUT)/ref_alpha.o
	$(CXX) -shared -o $@ $(OUT)/predicates.o $(OUT)/ref_pred.o $(OUT)/ref_alpha.o

$(OUT)/ga_%.o: $(ALPHA)/%.cu
	mkdir -p $(OUT)
	$(NVCC) $(NVFLAGS) -I$(REF)/gpudt -I$(ALPHA) -c $< -o $@

$(OUT)/ref_alpha_gpu.o: ref_alpha_gpu.cu
	mkdir -p $(OUT)
	$(NVCC) $(NVFLAGS) -I$(REF)/gpudt -I$(ALPHA) -c $< -o $@

$(OUT)/librefalpha.so: $(OUT)/ga_Alpha_Shapes_2D.o $(OUT)/ga_kernel.o $(OUT)/ga_headers.o $(OUT)/ref_alpha_gpu.o
	$(NVCC) -shared -gencode arch=compute_100a,code=sm_100a -o $@ $^

clean:
	rm -rf $(OUT)

.PHONY: all clean
