// Forwarding header at the reference's include path; the classes live in vanguard_shim.h.
#pragma once
#include "../../vanguard_shim.h"
