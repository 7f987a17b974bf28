# Compiles the reference's C API test file (read where it lies, unmodified) with the driver
# tests/c_api/ref_cases_main.c into tests/c_api/_ref/ref_c_api_cases, linked against this
# library (libcuopt_b200.so) through this repository's cuopt_c.h.  Test infrastructure: run where
# the reference tree is available; the binary is not committed.
#   make -f tests/c_api/ref_cases.mk REF=<reference project root>
REF  ?= /root/reference
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
ROOT := $(abspath $(HERE)/../..)
CC   := $(shell test -x /usr/bin/gcc && echo /usr/bin/gcc || echo gcc)
CUDA ?= /usr/local/cuda
OUT  := $(HERE)_ref
SRC  := $(REF)/cpp/tests/linear_programming/c_api_tests/c_api_test.c

$(OUT)/ref_c_api_cases: $(SRC) $(HERE)ref_cases_main.c $(ROOT)/cuopt_b200/libcuopt_b200.so
	mkdir -p $(OUT)
	$(CC) -std=gnu11 -O2 -w -I$(ROOT)/include -I$(CUDA)/include \
	  -I$(REF)/cpp/tests/linear_programming/c_api_tests \
	  $(SRC) $(HERE)ref_cases_main.c -o $@ \
	  -L$(ROOT)/cuopt_b200 -lcuopt_b200 -Wl,-rpath,'$$ORIGIN/../../../cuopt_b200' -lm
