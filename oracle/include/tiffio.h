/* tiffio.h -- types-only stand-in for libtiff (oracle build only).
 * deconwolf's fim_tiff.h includes <tiffio.h> for the TIFF handle type in its
 * prototypes; the oracle never reads or writes TIFF files, so an opaque type
 * is all that is needed.  libtiff is not installed here. */
#ifndef ORACLE_TIFFIO_STUB_H
#define ORACLE_TIFFIO_STUB_H
#include <stdint.h>
typedef struct oracle_tiff_s TIFF;
typedef uint32_t ttag_t;
typedef int64_t tmsize_t;
#endif
