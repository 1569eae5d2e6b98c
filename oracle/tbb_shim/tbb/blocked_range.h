/* Forwards to the single TBB stand-in header (oracle test infrastructure). */
#include "tbb.h"
