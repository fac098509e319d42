# Compiles the reference's own miniqmc driver, with the three libraries it
# links (qmcutil, qmcbase, qmcwfs: the source lists of src/CMakeLists.txt and
# src/QMCWaveFunctions/CMakeLists.txt), into oracle/_ref/ with the
# reference's GNU Release flags (CMakeLists.txt CMAKE_CXX_STANDARD 11;
# CMake/GNUCompilers.cmake: -fopenmp -fomit-frame-pointer -finline-limit=1000
# -fstrict-aliasing -funroll-all-loops -ffast-math; Release -O3 -DNDEBUG).
# The result is the timed CPU baseline of bench.py (--impl reference and the
# cpu_baseline field).  It is not the reference's CMake build: this Makefile,
# the hand-written oracle/ref_miniqmc_config.h for config.h, an empty
# git-rev.h, and the image's OpenBLAS (the BLAS/LAPACK the reference links,
# shipped in the opencv wheel) with an rpath to its directory (DT_RPATH, so
# that it also finds the libgfortran beside it).  The reference's
# -march=native becomes two fixed targets, x86-64-v3 (AVX2, FMA) and
# x86-64-v4 (AVX-512), because the binaries are built here and run on the GPU
# host; bench.py runs the widest one that host supports.  Each in FP64 (the
# default build) and in the reference's mixed precision
# (QMC_MIXED_PRECISION=1).  Without the reference tree every target is
# skipped.
MINIQMC_REFERENCE ?= /root/reference
REF := $(MINIQMC_REFERENCE)/src
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)_ref
REF_CXX ?= $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
PURELIB := $(shell python3 -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')
BLASDIR := $(PURELIB)/opencv_python_headless.libs
BLAS := $(firstword $(wildcard $(BLASDIR)/libopenblasp-*.so))
FLAGS := -O3 -DNDEBUG -std=c++11 -fopenmp -fomit-frame-pointer -finline-limit=1000 -fstrict-aliasing \
         -funroll-all-loops -ffast-math -Wno-deprecated -w -Drestrict=__restrict__ -D__forceinline=inline \
         -DHAVE_CONFIG_H -DADD_ -include cstdint -I$(OUT)/miniqmc_include -I$(REF)
SRCS := $(REF)/Drivers/miniqmc.cpp \
        $(REF)/QMCWaveFunctions/WaveFunction.cpp $(REF)/QMCWaveFunctions/SPOSet_builder.cpp \
        $(REF)/QMCWaveFunctions/DiracDeterminant.cpp $(REF)/QMCWaveFunctions/DiracDeterminantRef.cpp \
        $(REF)/Particle/VirtualParticleSet.cpp $(REF)/Particle/ParticleSet.cpp $(REF)/Particle/ParticleSet.BC.cpp \
        $(REF)/Particle/DistanceTableAA.cpp $(REF)/Particle/DistanceTableAB.cpp \
        $(REF)/Particle/ParticleSet_builder.cpp \
        $(REF)/Utilities/SpeciesSet.cpp $(REF)/Utilities/InfoStream.cpp $(REF)/Utilities/OutputManager.cpp \
        $(REF)/Utilities/Communicate.cpp $(REF)/Utilities/NewTimer.cpp $(REF)/Utilities/XMLWriter.cpp \
        $(REF)/Utilities/tinyxml/tinyxml2.cpp $(REF)/Utilities/qmcpack_version.cpp
LIBS := -L$(BLASDIR) -l:$(notdir $(BLAS)) -Wl,--disable-new-dtags -Wl,-rpath,$(BLASDIR) \
        -Wl,-rpath-link,$(BLASDIR) -lm
BINS := $(OUT)/miniqmc_v3 $(OUT)/miniqmc_v4 $(OUT)/miniqmc_mixed_v3 $(OUT)/miniqmc_mixed_v4

ifeq ($(wildcard $(REF)/Drivers/miniqmc.cpp),)
all:
	@echo "reference tree not found (set MINIQMC_REFERENCE): reference miniqmc not built"
else ifeq ($(BLAS),)
all:
	@echo "OpenBLAS not found under $(BLASDIR): reference miniqmc not built"
else
all: $(BINS)
endif

$(OUT)/miniqmc_include/config.h: $(HERE)ref_miniqmc_config.h
	mkdir -p $(OUT)/miniqmc_include
	cp $< $@
	touch $(OUT)/miniqmc_include/git-rev.h

$(OUT)/miniqmc_v3: $(OUT)/miniqmc_include/config.h
	$(REF_CXX) $(FLAGS) -march=x86-64-v3 -o $@ $(SRCS) $(LIBS)
$(OUT)/miniqmc_v4: $(OUT)/miniqmc_include/config.h
	$(REF_CXX) $(FLAGS) -march=x86-64-v4 -o $@ $(SRCS) $(LIBS)
$(OUT)/miniqmc_mixed_v3: $(OUT)/miniqmc_include/config.h
	$(REF_CXX) $(FLAGS) -DQMC_REF_MIXED -march=x86-64-v3 -o $@ $(SRCS) $(LIBS)
$(OUT)/miniqmc_mixed_v4: $(OUT)/miniqmc_include/config.h
	$(REF_CXX) $(FLAGS) -DQMC_REF_MIXED -march=x86-64-v4 -o $@ $(SRCS) $(LIBS)

clean:
	rm -rf $(OUT)/miniqmc_* $(OUT)/miniqmc_include

.PHONY: all clean
