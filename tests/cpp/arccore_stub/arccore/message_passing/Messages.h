// Stand-in for Arccore's <arccore/message_passing/Messages.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
