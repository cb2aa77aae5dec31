# Compiles a few of the reference's own C sources, read where they lie under the
# reference checkout (never copied), into oracle/_ref/ as shared libraries the
# oracle tests use as pins.  The Fortran production path cannot be built here
# (no Fortran compiler; the external libpvn build include is absent).
#   libjkref_alt.so : src/alt/wpqb.c (record comparator + greedy selection, qsort
#                     build without OpenMP), src/alt/j2apq.c (row-cyclic pairs) and
#                     src/alt/tweight.c (extended-precision trigonometric pair weight, with
#                     the project's plain-double entry points of ref_tw.c)
#   libjkref_var.so : src/var/qtransf.c, src/var/xtransf.c (80-bit 2x2 HSVDs)
#   libjkref_cutils.so : src/var/shared/cutils.c (x87 extended-precision HYPOT, DASUM2, DASUM4)
# wpqb.c keeps its selection count in the padding bytes of an 80-bit long double
# (a union) and then stores to the long double; an optimising build may drop the
# last count increment as a dead store, so the alt library is built at -O0.
# Usage: make -f ref.mk [REF=path/to/the/reference/checkout]
# By default the checkout is the repository's sibling directory `reference`.
REF ?= $(abspath $(CURDIR)/../../reference)
OUT := _ref
CC := gcc
CFLAGS := -std=gnu18 -fno-strict-aliasing -fPIC -shared -D_GNU_SOURCE -w

all: $(OUT)/libjkref_alt.so $(OUT)/libjkref_var.so $(OUT)/libjkref_cutils.so

$(OUT)/libjkref_alt.so: $(REF)/src/alt/wpqb.c $(REF)/src/alt/j2apq.c $(REF)/src/alt/tweight.c $(REF)/src/alt/common.c ref_tw.c
	mkdir -p $(OUT)
	$(CC) $(CFLAGS) -O0 -I$(REF)/src/alt -o $@ $^ -lm

$(OUT)/libjkref_var.so: $(REF)/src/var/qtransf.c $(REF)/src/var/xtransf.c $(REF)/src/var/common.c
	mkdir -p $(OUT)
	$(CC) $(CFLAGS) -O2 -DUSE_EXTENDED -I$(REF)/src/var -o $@ $^ -lm

$(OUT)/libjkref_cutils.so: $(REF)/src/var/shared/cutils.c
	mkdir -p $(OUT)
	$(CC) $(CFLAGS) -O2 -I$(REF)/src/var/shared -o $@ $^ -lm

clean:
	rm -rf $(OUT)

.PHONY: all clean
