# Compiles the reference's CPU dual simplex from its unmodified sources (read where they lie) with
# the stand-in headers of oracle/ref_shims and the driver oracle/ref_dual_simplex_main.cpp into
# oracle/_ref/ref_dual_simplex.  Test infrastructure: run where the reference tree is available
# (REF=<reference project root>); the binary is not committed.
#   make -C oracle ref REF=<reference project root>
REF  ?= /root/reference
CXX  := $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT  := $(HERE)_ref
OBJ  := $(OUT)/obj
SRCS := $(sort $(wildcard $(REF)/cpp/src/dual_simplex/*.cpp)) $(REF)/cpp/src/utilities/work_unit_scheduler.cpp
OBJS := $(patsubst %.cpp,$(OBJ)/%.o,$(notdir $(SRCS))) $(OBJ)/ref_dual_simplex_main.o
FLAGS := -std=c++20 -O3 -DNDEBUG -fopenmp -w -I$(HERE)ref_shims -I$(REF)/cpp/src -I$(REF)/cpp/include \
         -include utilities/logger.hpp

all: $(OUT)/ref_dual_simplex

$(OBJ)/%.o: $(REF)/cpp/src/dual_simplex/%.cpp | $(OBJ)
	$(CXX) $(FLAGS) -c $< -o $@
$(OBJ)/work_unit_scheduler.o: $(REF)/cpp/src/utilities/work_unit_scheduler.cpp | $(OBJ)
	$(CXX) $(FLAGS) -c $< -o $@
$(OBJ)/ref_dual_simplex_main.o: $(HERE)ref_dual_simplex_main.cpp | $(OBJ)
	$(CXX) $(FLAGS) -c $< -o $@
# The MIP entry points of solve.cpp reference branch-and-bound code that is not compiled; the
# dual simplex never calls them.
$(OUT)/ref_dual_simplex: $(OBJS)
	$(CXX) -fopenmp -o $@ $(OBJS) -Wl,--unresolved-symbols=ignore-in-object-files
$(OBJ):
	mkdir -p $@

.PHONY: all
