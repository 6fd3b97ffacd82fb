/*
 * ref_shim.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Prepended (by oracle/build.py) to the reference's OpenCL C kernel sources
 * so they compile as C on the host: the size #defines of
 * src/sodeclmgr.cpp:379-430 become process globals (see oracle_prelude.h)
 * and get_global_id(0) becomes the orbit index the host loop in
 * ref_driver.c sets before each call.
 */
#ifndef SODECL_REF_SHIM_H
#define SODECL_REF_SHIM_H
#include "oracle_prelude.h"
extern _Thread_local long g_ref_gid;
#define get_global_id(dim) ((int)g_ref_gid)
#endif
