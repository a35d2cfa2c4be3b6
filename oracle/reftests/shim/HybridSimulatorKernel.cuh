// Stand-in for the reference header of the same name: the whole restated
// API lives in refapi.h.
#pragma once
#include "refapi.h"
