/* The tag16h5 family in the upstream API (tag16h5.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tag16h5_create(void);
void tag16h5_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
