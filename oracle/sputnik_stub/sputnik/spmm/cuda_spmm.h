// Test-infrastructure stub (see ../sputnik.h).
#pragma once
#include "../sputnik.h"
