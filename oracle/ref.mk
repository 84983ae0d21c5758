# Builds the reference's own CPU primitives (test infrastructure only) from
# their sources where they lie, into oracle/_ref/libpfsf_ref.so, so the
# library's host exports can be checked against them bit for bit.
#
#   make -C oracle -f ref.mk
#
# Only the CPU translation units are used (compute/, ext/, trace/, diag/,
# and solver/amg_builder.cpp): they need no Vulkan and no generated code.  Compiled without FMA
# contraction and without -march, like this library's host code; the
# reference's own build adds -march=x86-64-v3, whose FMA contraction the Java
# side it mirrors does not have.  -Bsymbolic keeps the library's calls to
# its own exports inside itself when it is loaded beside libpfsf.so.
# The reference checkout: PFSF_REFERENCE, else a directory named "reference"
# beside this repository.
PFSF_REFERENCE ?= $(abspath $(CURDIR)/../../reference)
REF ?= $(PFSF_REFERENCE)/L1-native/libpfsf
OUT := _ref
CXX ?= g++
CXXFLAGS := -O2 -std=c++17 -fPIC -ffp-contract=off -w -I$(REF)/include -DPFSF_ABI_VERSION_STRING='"1.5.0"'
SRCS := $(wildcard $(REF)/src/compute/*.cpp) $(REF)/src/ext/augmentation.cpp $(REF)/src/ext/hooks.cpp \
        $(REF)/src/ext/plan_dispatcher.cpp $(REF)/src/trace/ring_buffer.cpp $(REF)/src/diag/crash.cpp

all: $(OUT)/libpfsf_ref.so $(OUT)/libpfsf_ref_amg.so

$(OUT)/libpfsf_ref.so: $(SRCS)
	mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS) -shared -Wl,-Bsymbolic -o $@ $(SRCS) -lpthread

# the reference's aggregation builder (solver/amg_builder.cpp: standard C++
# only) behind a C entry point of this directory's own (ref_amg_shim.cpp)
$(OUT)/libpfsf_ref_amg.so: $(REF)/src/solver/amg_builder.cpp ref_amg_shim.cpp
	mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS) -I$(REF)/src/solver -shared -o $@ $^

clean:
	rm -rf $(OUT)
