// Device arithmetic of the field picked by field_select.h.
#pragma once
#include "../field_select.h"

#if defined(QF_FIELD_KB)
#include "fkb_dev.cuh"
#else
#include "f65521_dev.cuh"
#endif
