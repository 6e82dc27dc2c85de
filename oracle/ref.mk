# Builds the unmodified ProtoMol reference from its sources where they lie,
# with plain g++ (no cmake, no generated headers: HAVE_PACKAGE_H stays
# undefined, which ProtoMolApp.cpp supports).  Test infrastructure only:
# every output goes to oracle/_ref/, which git ignores.
#
#   make -f oracle/ref.mk -j8 REF=<ProtoMol checkout>
#
# Outputs
#   oracle/_ref/libProtoMol.a      every library TU except base/Lapack.cpp
#                                  (ill-formed in C++11+ and unused on this
#                                  path) and integrator/openMM (needs OpenMM)
#   oracle/_ref/protomol           the stock ProtoMol executable
#   oracle/_ref/protomol_exacterf  same, with the Ewald module compiled with
#                                  -DUSE_EWALD_EXACT_ERF (libm erfc)
#   oracle/_ref/pm_forcedump       oracle/ref_forcedump.cpp linked to the
#                                  library: evaluates named forces on a
#                                  given configuration and dumps FP64
#                                  forces / energies / virial
#
# The drop-in itself (the stock driver plus the GPU module) is built by
# protomol_b200/protomol_module/Makefile against this library build.

ifndef REF
$(error REF must name the ProtoMol source checkout)
endif
OUT     ?= oracle/_ref
CXX     ?= g++
CXXFLAGS_REF ?= -std=c++98 -O2 -w -fno-strict-aliasing
INC     := -I$(REF) -I$(REF)/protomol

SRCS := $(shell cd $(REF) && find protomol -name '*.cpp' \
          ! -path 'protomol/integrator/openMM/*' \
          ! -name 'Lapack.cpp' ! -name 'main.cpp' ! -name 'modules.cpp' | sort)
OBJS := $(patsubst %.cpp,$(OUT)/obj/%.o,$(SRCS))
EXACT_OBJ := $(OUT)/obj_exact/NonbondedFullElectrostaticForceModule.o

all: $(OUT)/protomol $(OUT)/protomol_exacterf $(OUT)/pm_forcedump

$(OUT)/obj/%.o: $(REF)/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC) -c $< -o $@

$(OUT)/obj/lapack_stub.o: oracle/ref_lapack_stub.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC) -c $< -o $@

$(EXACT_OBJ): $(REF)/protomol/module/NonbondedFullElectrostaticForceModule.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -DUSE_EWALD_EXACT_ERF $(INC) -c $< -o $@

$(OUT)/libProtoMol.a: $(OBJS) $(OUT)/obj/lapack_stub.o
	rm -f $@
	ar rcs $@ $^

$(OUT)/obj/app/main.o: $(REF)/protomol/main.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC) -c $< -o $@

$(OUT)/obj/app/modules.o: $(REF)/protomol/modules.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC) -c $< -o $@

$(OUT)/protomol: $(OUT)/obj/app/main.o $(OUT)/obj/app/modules.o $(OUT)/libProtoMol.a
	$(CXX) -o $@ $^

# The exact-erf object is linked first so its instantiation of the Ewald
# templates is the one the executable keeps.
$(OUT)/protomol_exacterf: $(OUT)/obj/app/main.o $(OUT)/obj/app/modules.o $(EXACT_OBJ) $(OUT)/libProtoMol.a
	$(CXX) -o $@ $(OUT)/obj/app/main.o $(OUT)/obj/app/modules.o $(EXACT_OBJ) \
	  -Wl,--allow-multiple-definition $(OUT)/libProtoMol.a

$(OUT)/obj/app/ref_forcedump.o: oracle/ref_forcedump.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC) -c $< -o $@

$(OUT)/pm_forcedump: $(OUT)/obj/app/ref_forcedump.o $(OUT)/obj/app/modules.o $(OUT)/libProtoMol.a
	$(CXX) -o $@ $^

.PHONY: all
