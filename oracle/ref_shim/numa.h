/* Test infrastructure only (oracle build).
 *
 * Minimal stand-in for libnuma's header so that the reference's
 * src/Format/HBDIAVector.cpp compiles unchanged without libnuma installed.
 * The reference calls numa_alloc_onnode only on its NUMA-unified-memory
 * vector path (src/Format/HBDIAVector.cpp:129-142), which the oracle never
 * takes; the definition in oracle/ref_harness.cpp reports the call and
 * returns NULL. */
#ifndef HBDIA_ORACLE_NUMA_SHIM_H
#define HBDIA_ORACLE_NUMA_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
void *numa_alloc_onnode(size_t size, int node);
#ifdef __cplusplus
}
#endif
#endif
