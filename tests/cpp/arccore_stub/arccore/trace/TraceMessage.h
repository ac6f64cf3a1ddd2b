// Stand-in for Arccore's <arccore/trace/TraceMessage.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
