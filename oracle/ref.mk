# Builds the unmodified CURC reference (curc + bsc executables) from the
# sources where they lie, into oracle/_ref/.  Test infrastructure only: the
# binaries are the checker (archive round trips through `curc -d`, golden
# archives from `curc -c` on a GPU machine) and the reference arm of bench.py.
#
#   make -f oracle/ref.mk REF=<root of the reference source tree>
#
# The reference's own CMake build is not used.  Deviations from it, all
# needed to build with gcc 13 / nvcc 12.9 and none changing behaviour:
#   * -include cstdint (Param.hpp uses uint8_t without including it);
#   * fast-lzma2 compiled from its C sources (the shipped .so is not used);
#   * no -march=native (the binary must run on other x86-64 hosts).
ifndef REF
$(error REF must name the root of the reference source tree)
endif
OUT ?= oracle/_ref
NVCC ?= nvcc
CXX := g++
CC := gcc
ARCH ?= -gencode arch=compute_100a,code=sm_100a

OBJ := $(OUT)/obj
TP := $(REF)/third_party
COPT := -O2 -m64 -fopenmp -DLIBBSC_OPENMP_SUPPORT
INC := -isystem $(TP) -include cstdint

FL2_SRC := $(wildcard $(TP)/fast-lzma2/*.c)
FL2_OBJ := $(patsubst $(TP)/fast-lzma2/%.c,$(OBJ)/fl2/%.o,$(FL2_SRC))
LZMA_C := LzmaEnc LzmaDec Alloc LzFindMt LzFind Ppmd7 Ppmd7Enc Ppmd7Dec Threads
LZMA_CXX := LzmaLib VarLenDNACoder helper
LZMA_OBJ := $(patsubst %,$(OBJ)/lzma/%.o,$(LZMA_C)) $(patsubst %,$(OBJ)/lzma/vl_%.o,$(LZMA_CXX))
BSC_CXX := bsc libbsc/adler32/adler32 libbsc/bwt/bwt libbsc/coder/qlfc/qlfc \
	libbsc/coder/qlfc/qlfc_model libbsc/coder/coder libbsc/filters/detectors \
	libbsc/filters/preprocessing libbsc/libbsc/libbsc libbsc/lzp/lzp libbsc/platform/platform
BSC_OBJ := $(patsubst %,$(OBJ)/bsc/%.o,$(BSC_CXX)) $(OBJ)/bsc/divsufsort.o
CURC_OBJ := $(OBJ)/main.o $(OBJ)/preprocess.o $(OBJ)/compress.o $(OBJ)/decompress.o $(OBJ)/fast_lzma2_helper.o

all: $(OUT)/curc $(OUT)/bsc $(OUT)/libcurc_coders.a

$(OBJ)/fl2/%.o: $(TP)/fast-lzma2/%.c
	@mkdir -p $(dir $@)
	$(CC) -O2 -pthread -fPIC -c $< -o $@

$(OBJ)/lzma/%.o: $(TP)/lzma/%.c
	@mkdir -p $(dir $@)
	$(CC) $(COPT) -fPIC -c $< -o $@

$(OBJ)/lzma/vl_%.o: $(TP)/lzma/VarLenDNACoder/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) -std=c++17 $(COPT) -fPIC $(INC) -c $< -o $@

$(OBJ)/bsc/divsufsort.o: $(TP)/libbsc/libbsc/bwt/divsufsort/divsufsort.c
	@mkdir -p $(dir $@)
	$(CC) $(COPT) -c $< -o $@

$(OBJ)/bsc/%.o: $(TP)/libbsc/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(COPT) -c $< -o $@

$(OBJ)/%.o: $(REF)/src/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) -std=c++17 $(COPT) -fPIC $(INC) -c $< -o $@

$(OBJ)/compress.o: $(REF)/src/compress.cu
	@mkdir -p $(dir $@)
	$(NVCC) -std=c++14 $(ARCH) --expt-extended-lambda -O3 -Xcompiler -O2,-fopenmp,-pthread $(INC) -c $< -o $@

$(OBJ)/decompress.o: $(REF)/src/decompress.cu
	@mkdir -p $(dir $@)
	$(NVCC) -std=c++14 $(ARCH) --expt-extended-lambda -O3 -Xcompiler -O2,-fopenmp,-pthread --pre-include cstdint -isystem $(TP) -c $< -o $@

$(OUT)/libfast-lzma2.a: $(FL2_OBJ)
	ar rcs $@ $^

# Coders only (fast-lzma2, LZMA SDK + PPMd7, VarLenDNACoder): lets the oracle
# write and read archives in the reference layout.
$(OUT)/libcurc_coders.a: $(FL2_OBJ) $(LZMA_OBJ) $(OBJ)/fast_lzma2_helper.o
	ar rcs $@ $^

$(OUT)/curc: $(CURC_OBJ) $(LZMA_OBJ) $(OUT)/libfast-lzma2.a
	$(NVCC) $(ARCH) -o $@ $(CURC_OBJ) $(LZMA_OBJ) $(OUT)/libfast-lzma2.a -lgomp -lstdc++fs -lpthread

$(OUT)/bsc: $(BSC_OBJ)
	$(CXX) -o $@ $^ -lgomp -lpthread

.PHONY: all

# Golden-archive variant: same objects linked against the shared CUDA
# runtime, plus the zero-filling cudaMalloc shim (ref_zero_alloc.c).
golden: $(OUT)/curc_shared $(OUT)/libzero_alloc.so

$(OUT)/curc_shared: $(CURC_OBJ) $(LZMA_OBJ) $(OUT)/libfast-lzma2.a
	$(NVCC) $(ARCH) -cudart shared -o $@ $(CURC_OBJ) $(LZMA_OBJ) $(OUT)/libfast-lzma2.a -lgomp -lstdc++fs -lpthread

$(OUT)/libzero_alloc.so: oracle/ref_zero_alloc.c
	$(CC) -O2 -shared -fPIC -o $@ $< -L$(CUDA_HOME)/lib64 -lcudart -ldl -lpthread

CUDA_HOME ?= /usr/local/cuda
.PHONY: golden
