# Builds the reference's CPU library (the FP64 oracle and the timed CPU
# baseline) straight from its sources with g++, without its own build system.
# Inputs are read in place under REF; every output lands in oracle/_ref/.
#   make -f oracle/ref.mk -j8 REF=<reference checkout>
# REF comes from the command line or $XTBLOOM_REFERENCE_SRC.  The BLAS/LAPACK
# the reference's eigensolver loads at run time is the OpenBLAS that ships
# inside the installed scipy wheel (LP64, scipy_-prefixed symbols), located
# through the Python interpreter on PATH.
REF      ?= $(XTBLOOM_REFERENCE_SRC)
OUT      ?= $(dir $(lastword $(MAKEFILE_LIST)))_ref
OPENBLAS ?= $(shell python3 -c 'import glob, os, scipy; d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs"); print((sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so"))) or [""])[0])')
ifeq ($(strip $(REF)),)
$(error set REF=<reference checkout> or XTBLOOM_REFERENCE_SRC)
endif

SRCS := src/api.cpp src/runtime/backend.cpp src/runtime/gfn2_cpu_execution.cpp \
  src/runtime/gfn2_plan.cpp src/runtime/model_plan.cpp src/runtime/model_registry.cpp \
  src/runtime/request.cpp src/runtime/result_owner.cpp src/runtime/validation.cpp \
  src/cpu_dispatch/features.cpp src/model/gfn2/mulliken_kernels_baseline.cpp \
  src/model/common/sto.cpp src/model/common/integrals.cpp src/model/common/scc_mixer.cpp \
  src/model/gfn2/eigensolver.cpp src/model/gfn2/periodic_embedding.cpp src/model/gfn2/es2.cpp \
  src/backends/common/gfn2_plan_schema.cpp src/model/gfn2/aes2.cpp src/model/gfn2/basis.cpp \
  src/model/gfn2/coordination.cpp src/model/gfn2/d4.cpp src/model/gfn2/es3.cpp \
  src/model/gfn2/external_point_charges.cpp src/model/gfn2/force.cpp src/model/gfn2/h0.cpp \
  src/model/gfn2/lattice.cpp src/model/gfn2/mulliken.cpp src/model/gfn2/mulliken_kernels.cpp \
  src/model/gfn2/repulsion.cpp src/model/gfn2/scc_driver.cpp src/model/gfn2/scc_mixer.cpp \
  src/model/gfn2/spin.cpp src/model/gfn2/wavefunction.cpp \
  src/model/gfn1/basis.cpp src/model/gfn1/coordination.cpp src/model/gfn1/d3.cpp \
  src/model/gfn1/es2.cpp src/model/gfn1/es3.cpp src/model/gfn1/external_point_charges.cpp \
  src/model/gfn1/force.cpp src/model/gfn1/h0.cpp src/model/gfn1/halogen.cpp \
  src/model/gfn1/mulliken.cpp src/model/gfn1/repulsion.cpp src/model/gfn1/scc_driver.cpp \
  src/model/gfn1/scc_mixer.cpp src/model/gfn1/spin.cpp src/model/gfn1/wavefunction.cpp \
  src/runtime/gfn1_cpu_execution.cpp

OBJS := $(patsubst %.cpp,$(OUT)/obj/%.o,$(SRCS))
CXXFLAGS := -std=c++17 -O2 -fPIC -fvisibility=hidden -fvisibility-inlines-hidden \
  -I$(OUT)/gen -I$(REF) -I$(REF)/include -I$(REF)/src \
  -DXTBLOOM_BUILDING_LIBRARY '-DXTBLOOM_CONFIGURED_CPU_LINALG_RUNTIME="$(OPENBLAS)"'

all: $(OUT)/libxtbloom_ref.so

$(OUT)/gen/xtbloom/version.h:
	@mkdir -p $(dir $@)
	printf '#ifndef XTBLOOM_VERSION_H\n#define XTBLOOM_VERSION_H\n#define XTBLOOM_VERSION_MAJOR 0\n#define XTBLOOM_VERSION_MINOR 1\n#define XTBLOOM_VERSION_PATCH 0\n#define XTBLOOM_VERSION_STRING "0.1.0-oracle"\n#endif\n' > $@

$(OUT)/obj/%.o: $(REF)/%.cpp $(OUT)/gen/xtbloom/version.h
	@mkdir -p $(dir $@)
	g++ $(CXXFLAGS) -c $< -o $@

$(OUT)/libxtbloom_ref.so: $(OBJS)
	g++ -shared -o $@ $(OBJS) -Wl,--version-script=$(REF)/cmake/xtbloom.map -lpthread -ldl

.PHONY: all
