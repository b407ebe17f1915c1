/* ne_oracle.h -- TEST INFRASTRUCTURE ONLY: the C restatement of the
 * reference's World::step() used as a checker.  Never linked into the product.
 * Same entry points as the reference shim (oracle/ref_shim.cpp), prefix
 * "neport_", over the POD structs of include/ne_cuda.h. */
#ifndef NE_ORACLE_H
#define NE_ORACLE_H

#include <stdint.h>

#include "ne_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

void* neport_create(const NeWorldParams* p, const NeBodyArrays* b);
void neport_destroy(void* h);
void neport_set_params(void* h, const NeWorldParams* p);
void neport_reset_warm_cache(void* h);
void neport_step(void* h, uint32_t nsteps);
void neport_get_state(void* h, NeBodyArrays* out);
uint64_t neport_pairs(void* h, uint32_t* pi, uint32_t* pj, uint64_t cap);
uint64_t neport_contacts(void* h, NeContactArrays* out, uint64_t cap);
void neport_islands(void* h, uint32_t* label, uint32_t n);

#ifdef __cplusplus
}
#endif

#endif /* NE_ORACLE_H */
