// APTPhaseField.h — for callers written against the reference's headers
// (3DgrainMPI/APTPhaseField.h): the driver's APTPhaseField (phase_field.h) under the reference's name.
#pragma once
#include "MPIsetting.h"
#include "../phase_field.h"
using cupf_host::APTPhaseField;
