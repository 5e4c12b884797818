/* Test infrastructure only: linked into the parity build of the reference (oracle/Makefile) with
 * -Wl,-Bsymbolic-functions, so the reference's own calls of expf and powf (its ground friction,
 * static_world.cpp:41-44) take the oracle's portable functions instead of libm's. See orc_math.h. */
#include "orc_math.h"

float expf(float x) { return orc_expf(x); }
float powf(float x, float y) { return orc_powf(x, y); }
