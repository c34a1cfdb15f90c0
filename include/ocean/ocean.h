/* oceanlib-b200 - the reference's C header path (include/ocean/ocean.h of
 * DarshanVShah/oceanlib).
 *
 * A C or C++ translation unit written against the reference includes
 * "ocean/ocean.h"; here that header is the B200 library's C ABI, whose first
 * part re-declares every reference entry point with the same names, struct
 * layouts, status codes and NULL-handle behaviour (ocean_b200.h Part 1),
 * followed by the device extensions (Part 2). Plain C89-compatible
 * declarations throughout.
 */
#ifndef OCEANLIB_OCEAN_H
#define OCEANLIB_OCEAN_H

#include "../ocean_b200.h"

#endif /* OCEANLIB_OCEAN_H */
