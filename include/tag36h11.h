/* The tag36h11 family in the upstream API (tag36h11.h of the reference): the codes are
   the library's built-in table; destroy frees only what create allocated. */
#pragma once
#include "apriltag.h"

#ifdef __cplusplus
extern "C" {
#endif

apriltag_family_t *tag36h11_create(void);
void tag36h11_destroy(apriltag_family_t *tf);

#ifdef __cplusplus
}
#endif
