/* Build shim for compiling HiFlow3's lmp CPU sources outside their CMake
 * build (test infrastructure only: used by oracle/ref/Makefile to produce the
 * reference CPU checker under oracle/_ref/).
 *
 * Stands in for the CMake-generated config.h (template src/config.h.in).
 * Only the switches the lmp CPU NAIVE/OPENMP path reads are defined; no
 * CUDA/OpenCL/MKL/CBLAS backends are enabled. */
#ifndef B200LA_ORACLE_SHIM_CONFIG_H
#define B200LA_ORACLE_SHIM_CONFIG_H

#define WITH_OPENMP 1

const int DEBUG_LEVEL = 0;

#endif
