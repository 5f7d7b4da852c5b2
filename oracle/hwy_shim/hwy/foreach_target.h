// Single-target stand-in: the including file is compiled exactly once,
// with HWY_TARGET_TOGGLE left undefined, so the reference -inl headers take
// their first-inclusion branch.
#include "highway.h"
