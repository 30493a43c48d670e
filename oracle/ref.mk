# Compiles the reference's C matrix generator from its own sources, where
# they lie, into oracle/_ref/ref_poisson (test infrastructure: it produces
# the known-answer Poisson fixtures under tests/golden/).  Nothing is copied
# out of the reference tree.  Usage: make -f oracle/ref.mk REF=/path/to/cel_v3
# (REF is the root of a hpcdkhab/cel_v3 checkout; it has no default)
ifeq ($(strip $(REF)),)
$(error REF is not set: make -f oracle/ref.mk REF=/path/to/cel_v3)
endif
OUT := $(dir $(lastword $(MAKEFILE_LIST)))_ref
SRC := $(REF)/src/base
REF_SOURCES := $(SRC)/cel_sparce_matrix_coo_interface.c $(SRC)/cel_discretisation.c \
  $(SRC)/cel_discretisation_poisson_3d.c $(SRC)/cel_domain_3d.c $(SRC)/cel_sort.c \
  $(SRC)/cel_sparse_matrix_coo.c $(SRC)/cel_vector.c
DRIVER := $(dir $(lastword $(MAKEFILE_LIST)))ref_poisson_main.c

all: $(OUT)/ref_poisson

$(OUT)/ref_poisson: $(REF_SOURCES) $(DRIVER)
	mkdir -p $(OUT)
	/usr/bin/gcc -std=gnu99 -O2 -ffp-contract=off -w -I$(REF)/src/include/base \
	  -o $@ $(DRIVER) $(REF_SOURCES) -lm

.PHONY: all
