// Picks the field of a backend translation unit: F65521^8 with signed 8-bit
// weights by default, KoalaBear^4 with signed 16-bit payloads when QF_FIELD_KB
// is defined.  QFD_NS names the namespace of the field's device code, QFB_NS
// that of its host backend.
#pragma once
#include <cstdint>

#include "host/field65521.h"
#include "host/fieldkb.h"

#if defined(QF_FIELD_KB)
#define QFD_NS qfdkb
#define QFB_NS qfgkb
namespace qfgkb {
using F = ::qf::Kb4;
using W = int16_t;  // one signed payload
}
#else
#define QFD_NS qfd
#define QFB_NS qfg
namespace qfg {
using F = ::qf::Fp8;
using W = int8_t;  // one signed weight
}
#endif
