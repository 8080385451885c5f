/* The tagCircle49h12 family in the upstream API (tagCircle49h12.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tagCircle49h12_create(void);
void tagCircle49h12_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
