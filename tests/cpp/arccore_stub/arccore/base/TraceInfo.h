// Stand-in for Arccore's <arccore/base/TraceInfo.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
