/* Include path the reference's callers use (#include "grrt/api.h"); the
 * declarations live in grrt_api.h. */
#ifndef GRRT_B200_COMPAT_API_H
#define GRRT_B200_COMPAT_API_H
#include "../grrt_api.h"
#endif
