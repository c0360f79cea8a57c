// Types.cpp -- storage of SimTools::EPSILON (source/Types.cpp:9).  Zero-
// initialised as in the reference, where only some case set-ups assign it.
#include "Types.h"

double SimTools::EPSILON;
