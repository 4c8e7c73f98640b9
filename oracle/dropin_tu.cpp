// Test infrastructure: compiles include/rr_ri.hpp (the C++ overloads over librr_ri) as the one
// translation unit that replaces the reference's RI .cpp files, so that the reference's own SCF
// loops and bridge (oracle/_ref/librrref_dropin.so) run on the GPU path unchanged.
#define RR_RI_DROPIN_DEFINE
#include "rr_ri.hpp"
