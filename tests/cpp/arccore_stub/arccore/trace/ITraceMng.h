// Stand-in for Arccore's <arccore/trace/ITraceMng.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
