/* Declaration-only stand-in for the SPOOLES header misc.h (the SPOOLES
 * sources are not available): the entry points the reference calls are
 * declared in spooles_types.h and implemented in spooles_shim.cpp. */
#include "spooles_types.h"
