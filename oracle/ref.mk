# Builds the reference (front end, operators, codec, CLI) for the CPU from its own
# sources where they lie, into oracle/_ref/alenka_ref. Thrust's OpenMP device system
# stands in for CUDA; oracle/ref_shim supplies host versions of the CUDA runtime calls,
# Thrust 2.x's removed pinned_allocator, and the three moderngpu primitives the
# reference calls (moderngpu is not vendored with it). No reference source is copied;
# objects go to oracle/_ref/obj only. Test infrastructure and CPU baseline only.
#   make -f oracle/ref.mk REF=<reference checkout>
REF ?= /root/reference
HERE := $(dir $(lastword $(MAKEFILE_LIST)))
SHIM := $(abspath $(HERE)ref_shim)
OUT := $(abspath $(HERE)_ref)
CUDA_INC ?= /usr/local/cuda/include
GCC_LIB ?= /usr/lib/gcc/x86_64-linux-gnu/13
CXXFLAGS = -std=c++14 -O2 -w -fopenmp -x c++ -DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_OMP \
  -I$(SHIM) -I$(CUDA_INC) -include $(SHIM)/cuda_host_shim.h -include algorithm -include iostream
SRCS = bison cm operators select merge filter zone_map MurmurHash2_64 atof \
  strings_join strings_sort_host strings_sort_device main
OBJS = $(addprefix $(OUT)/obj/,$(addsuffix .o,$(SRCS)) callbacks.o)

$(OUT)/alenka_ref: $(OBJS)
	g++ -fopenmp -o $@ $(OBJS) -L$(GCC_LIB) -lgomp -lpthread

$(OUT)/obj/%.o: $(REF)/%.cu $(wildcard $(SHIM)/*.h $(SHIM)/moderngpu/src/moderngpu/*.hxx)
	@mkdir -p $(OUT)/obj
	g++ $(CXXFLAGS) -c $< -o $@

$(OUT)/obj/callbacks.o: $(REF)/callbacks.c
	@mkdir -p $(OUT)/obj
	gcc -O2 -w -c $< -o $@

# The reference's own front end (the generated parser bison.cu + lex.yy.c, main.cu and
# callbacks.c, compiled above, unchanged) linked against this repository's library in
# place of the reference's operators: the reference CLI running scripts on the engine.
LIB := $(abspath $(HERE)../alenka_b200/libalenka_b200.so)
FRONT_LDFLAGS = -Wl,-rpath,'$$ORIGIN/../../alenka_b200' -fopenmp -L$(GCC_LIB) -lgomp -lpthread
FRONT_OBJS = $(OUT)/obj/bison.o $(OUT)/obj/atof.o $(OUT)/obj/callbacks.o
$(OUT)/alenka_frontend: $(FRONT_OBJS) $(OUT)/obj/main.o $(LIB)
	g++ -o $@ $(FRONT_OBJS) $(OUT)/obj/main.o $(LIB) $(FRONT_LDFLAGS)

# The same parser's first pass only, printing what the library's emit_* boundary captured
$(OUT)/frontend_dump: $(HERE)frontend_dump.cpp $(FRONT_OBJS) $(LIB)
	g++ -std=c++14 -O1 -o $@ $< $(FRONT_OBJS) $(LIB) $(FRONT_LDFLAGS)

frontend: $(OUT)/alenka_frontend $(OUT)/frontend_dump
.PHONY: frontend
