/* Include path of the reference's parameter types (#include "grrt/types.h");
 * GRRTParams and the enums live in grrt_api.h. */
#ifndef GRRT_B200_COMPAT_TYPES_H
#define GRRT_B200_COMPAT_TYPES_H
#include "../grrt_api.h"
#endif
