// AllocateAligned lives in highway.h in this stand-in.
#include "highway.h"
