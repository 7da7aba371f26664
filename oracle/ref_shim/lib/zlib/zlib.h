/* Build shim for compiling the reference's sources offline: the reference
 * includes "../lib/zlib/zlib.h" (a vendored zlib build); the system zlib is
 * used instead.  Only affects BGZF output bytes, never the alignment path. */
#include <zlib.h>
