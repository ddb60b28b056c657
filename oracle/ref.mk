# Builds oracle/_ref/libref.so from the reference's own sources, where they lie
# (never copied into this repository).  Test infrastructure only: the CPU tests
# use it to pin the oracle's exact arithmetic against the reference's
# predicates.  Needs only g++; the reference's cmake/GL build is not used.
#
#   gpudt/predicates.cpp              host orient2d / incircle (Shewchuk, adaptive)
#   gpudt/AlphaShape/predicates.h     alpha birth times, attached test, exact
#                                     squared-radius comparisons (host-compiled)
REF ?= /root/reference
CXX ?= g++
FLAGS = -O2 -fPIC -ffp-contract=off -fno-fast-math -w
OUT = _ref

all: $(OUT)/libref.so

$(OUT)/libref.so: ref_pred.cpp ref_alpha.cpp
	mkdir -p $(OUT)
	$(CXX) $(FLAGS) -I$(REF)/gpudt -c $(REF)/gpudt/predicates.cpp -o $(OUT)/predicates.o
	$(CXX) $(FLAGS) -I$(REF)/gpudt -c ref_pred.cpp -o $(OUT)/ref_pred.o
	$(CXX) $(FLAGS) -I$(REF)/gpudt -c ref_alpha.cpp -o $(OUT)/ref_alpha.o
	$(CXX) -shared -o $@ $(OUT)/predicates.o $(OUT)/ref_pred.o $(OUT)/ref_alpha.o

clean:
	rm -rf $(OUT)

.PHONY: all clean
