/* Umbrella header, as the reference's algebra/include/midapack.h. */
#ifndef MDP_DROPIN_MIDAPACK_H
#define MDP_DROPIN_MIDAPACK_H
#include "mapmat.h"
#include "toeplitz.h"
#endif
