// march_fast.cu — the persistent march of march.cu built with approximate
// division and square root (-prec-div=false -prec-sqrt=false): the default
// march of the ray-queue schedule.  The march only produces visibility (the
// reservoirs are final before it runs), so this changes radiance within the
// parity tolerance and no selection.
#define IRT_MARCH_FAST 1
#include "march.cu"
