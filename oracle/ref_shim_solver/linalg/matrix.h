/* host shim: see linalg.h in this directory */
#pragma once
#include "linalg/linalg.h"
