// Stand-in (oracle test infrastructure): see core.h.
#pragma once
#include "core.h"
