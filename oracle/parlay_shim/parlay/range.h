// Forwarding header of the project parlay shim (test infrastructure).
#pragma once
#include "shim_core.h"
