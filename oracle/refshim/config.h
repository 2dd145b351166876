// config.h -- stand-in for the header the reference's CMake generates from
// include/config.h.in (it defines only SOURCE_DIR).  TEST INFRASTRUCTURE
// ONLY: used by oracle/Makefile to compile the reference's solver sources
// in place for the reference pin.
#ifndef PXP_REFSHIM_CONFIG_H
#define PXP_REFSHIM_CONFIG_H
#define SOURCE_DIR ""
#endif
