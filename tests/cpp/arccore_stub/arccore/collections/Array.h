// Stand-in for Arccore's <arccore/collections/Array.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
