// Stand-in for Arccore's <arccore/message_passing/Request.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
