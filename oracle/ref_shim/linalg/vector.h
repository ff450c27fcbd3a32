/* host shim: see algo/types.h in this directory */
#pragma once
#include "algo/types.h"
