// The field-specific C ABI bodies compiled for KoalaBear^4 with signed 16-bit
// payloads (exported as qfgkb::kFieldApi).
#define QF_FIELD_KB 1
#include "capi_field.cu"
