/* Correctly rounded single-precision trig for the reference build.

   Test infrastructure only: force-included (-include) when the unmodified
   reference detector is compiled into oracle/_ref. The reference's edge
   refinement calls atan2f, cosf and sinf (fast/decode.c:740-744); its
   committed golden vectors were produced with a libm whose float trig is
   correctly rounded. glibc's float versions are not, so here each one is
   evaluated in double and rounded once to float, which is the correctly
   rounded result except for arguments within about 2^-29 relative of a
   rounding boundary. */
#ifndef AT_TRIG_CR_H
#define AT_TRIG_CR_H
#include <math.h>
static inline float at_cr_atan2f(float y, float x) { return (float)atan2((double)y, (double)x); }
static inline float at_cr_cosf(float x) { return (float)cos((double)x); }
static inline float at_cr_sinf(float x) { return (float)sin((double)x); }
#define atan2f at_cr_atan2f
#define cosf at_cr_cosf
#define sinf at_cr_sinf
#endif
