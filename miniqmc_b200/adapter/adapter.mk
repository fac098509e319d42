# Links the reference's own drivers, unmodified, against libqmcgpu through
# the adapter classes (qmcgpu_adapter.hpp):
#   ../bin/ref_miniqmc            Drivers/miniqmc.cpp
#   ../bin/ref_miniqmc_sync_move  Drivers/miniqmc_sync_move.cpp
#   ../bin/check_spo_gpu          the reference's SPO set against SPOSetGpu
# Each binary is the driver's source and the reference's particle, SPO
# builder and utility sources (the qmcutil / qmcbase source lists of
# src/CMakeLists.txt), compiled with the reference's GNU Release flags
# (CMakeLists.txt, CMake/GNUCompilers.cmake) less -ffast-math and with
# -ffp-contract=off, plus the adapter in place of
# QMCWaveFunctions/WaveFunction.cpp.  The reference's DiracDeterminant,
# Jastrow and BLAS code is not linked: the wavefunction is the device's.
# With IEEE arithmetic and no fused multiply-adds the drivers' host values
# (electron positions from build_els, BoxMuller2 normals, the NLPP
# distances and sphere points) are the ones any other IEEE build of the
# same streams gives, and the adapter's move displacements stay exact.
# Without the reference tree the targets are skipped.
MINIQMC_REFERENCE ?= /root/reference
REF := $(MINIQMC_REFERENCE)/src
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
PKG := $(abspath $(HERE)..)
ROOT := $(abspath $(PKG)/..)
BIN := $(PKG)/bin
OBJ := $(PKG)/_build/adapter
REF_CXX ?= $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
COMMON := -std=c++11 -fopenmp -ffp-contract=off -w -Drestrict=__restrict__ -D__forceinline=inline -DHAVE_CONFIG_H -DADD_ \
          -include cstdint -I$(HERE)include -I$(REF)
REF_FLAGS := -O3 -DNDEBUG $(COMMON) -fomit-frame-pointer -finline-limit=1000 -fstrict-aliasing \
             -funroll-all-loops -march=x86-64-v3
ADAPTER_FLAGS := -O2 -DNDEBUG $(COMMON) -I$(ROOT)/include
REF_SRCS := Particle/VirtualParticleSet.cpp Particle/ParticleSet.cpp Particle/ParticleSet.BC.cpp \
            Particle/DistanceTableAA.cpp Particle/DistanceTableAB.cpp Particle/ParticleSet_builder.cpp \
            QMCWaveFunctions/SPOSet_builder.cpp \
            Utilities/SpeciesSet.cpp Utilities/InfoStream.cpp Utilities/OutputManager.cpp \
            Utilities/Communicate.cpp Utilities/NewTimer.cpp Utilities/XMLWriter.cpp \
            Utilities/tinyxml/tinyxml2.cpp Utilities/qmcpack_version.cpp
REF_OBJS := $(addprefix $(OBJ)/ref/,$(REF_SRCS:.cpp=.o))
ADAPTER_OBJS := $(OBJ)/qmcgpu_adapter.o $(OBJ)/qmcgpu_wavefunction.o
LIBS := -L$(PKG) -lqmcgpu -Wl,-rpath,'$$ORIGIN/..' -fopenmp -lm
BINS := $(BIN)/ref_miniqmc $(BIN)/ref_miniqmc_sync_move $(BIN)/check_spo_gpu

ifeq ($(wildcard $(REF)/Drivers/miniqmc.cpp),)
all:
	@echo "reference tree not found (set MINIQMC_REFERENCE): reference drivers on the device not built"
else
all: $(BINS)
endif

$(OBJ)/ref/%.o: $(REF)/%.cpp
	@mkdir -p $(dir $@)
	$(REF_CXX) $(REF_FLAGS) -c -o $@ $<

$(OBJ)/drivers/%.o: $(REF)/Drivers/%.cpp
	@mkdir -p $(dir $@)
	$(REF_CXX) $(REF_FLAGS) -c -o $@ $<

$(OBJ)/%.o: $(HERE)%.cpp $(HERE)qmcgpu_adapter.hpp $(ROOT)/include/qmcgpu.h
	@mkdir -p $(dir $@)
	$(REF_CXX) $(ADAPTER_FLAGS) -c -o $@ $<

$(BIN)/check_spo_gpu: $(OBJ)/check_spo_gpu.o $(REF_OBJS) $(ADAPTER_OBJS) $(PKG)/libqmcgpu.so
	@mkdir -p $(BIN)
	$(REF_CXX) -o $@ $< $(REF_OBJS) $(ADAPTER_OBJS) $(LIBS)

$(BIN)/ref_%: $(OBJ)/drivers/%.o $(REF_OBJS) $(ADAPTER_OBJS) $(PKG)/libqmcgpu.so
	@mkdir -p $(BIN)
	$(REF_CXX) -o $@ $< $(REF_OBJS) $(ADAPTER_OBJS) $(LIBS)

clean:
	rm -rf $(OBJ) $(BINS)

.PHONY: all clean
.SECONDARY:
