/* Library version; replaces iderex/cudec src/version.c:3-6. */
#include "cudec.h"

int cudec_version(void) {
    return CUDEC_VERSION_MAJOR * 10000 + CUDEC_VERSION_MINOR * 100 +
           CUDEC_VERSION_PATCH;
}
