# Compiles the reference's own sources (read-only, where MINIQMC_REFERENCE
# points) with the golden-dump drivers oracle/ref_harness.cpp and
# oracle/ref_det_harness.cpp into oracle/_ref/.  The determinant driver links
# the image's OpenBLAS (the BLAS/LAPACK the reference's DiracMatrix and
# DelayedUpdate call).  Without the reference tree the targets are skipped.
# Test infrastructure only: not the reference's CMake build, no external
# libraries; the hand-written oracle/ref_harness_config.h replaces the
# CMake-generated config.h.
MINIQMC_REFERENCE ?= /root/reference
REF := $(MINIQMC_REFERENCE)/src
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)_ref
REF_CXX ?= $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
# the reference's plain FP64 build flags (no -ffast-math)
FLAGS := -O2 -std=c++11 -fopenmp -ffp-contract=off -w -Drestrict=__restrict__ -DHAVE_CONFIG_H -DADD_ -D__forceinline=inline -fomit-frame-pointer -fstrict-aliasing -include cstdint -I$(OUT)/include -I$(REF)
SRCS := $(REF)/Particle/ParticleSet.cpp $(REF)/Particle/ParticleSet.BC.cpp \
        $(REF)/Particle/DistanceTableAA.cpp $(REF)/Particle/DistanceTableAB.cpp \
        $(REF)/Particle/ParticleSet_builder.cpp $(REF)/Utilities/SpeciesSet.cpp \
        $(REF)/Utilities/NewTimer.cpp $(REF)/Utilities/OutputManager.cpp \
        $(REF)/Utilities/InfoStream.cpp $(REF)/Utilities/XMLWriter.cpp \
        $(REF)/Utilities/tinyxml/tinyxml2.cpp

PURELIB := $(shell python3 -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')
BLASDIR := $(PURELIB)/opencv_python_headless.libs
BLAS := $(firstword $(wildcard $(BLASDIR)/libopenblasp-*.so))
BLASLIBS := -L$(BLASDIR) -l:$(notdir $(BLAS)) -Wl,--disable-new-dtags -Wl,-rpath,$(BLASDIR) \
            -Wl,-rpath-link,$(BLASDIR) -lm

ifeq ($(wildcard $(REF)/Particle/ParticleSet.cpp),)
all:
	@echo "reference tree not found (set MINIQMC_REFERENCE): golden-dump harness not built"
else ifeq ($(BLAS),)
all: $(OUT)/ref_harness
else
all: $(OUT)/ref_harness $(OUT)/ref_det_harness
endif

$(OUT)/include/config.h: $(HERE)ref_harness_config.h
	mkdir -p $(OUT)/include
	cp $< $@

$(OUT)/ref_harness: $(HERE)ref_harness.cpp $(OUT)/include/config.h
	$(REF_CXX) $(FLAGS) -o $@ $(HERE)ref_harness.cpp $(SRCS)

$(OUT)/ref_det_harness: $(HERE)ref_det_harness.cpp $(OUT)/include/config.h
	$(REF_CXX) $(FLAGS) -o $@ $(HERE)ref_det_harness.cpp $(SRCS) $(REF)/QMCWaveFunctions/DiracDeterminant.cpp \
	    $(BLASLIBS)

clean:
	rm -rf $(OUT)

.PHONY: all clean
