// PhaseField.h — for callers written against the reference's headers
// (3DgrainMPI/PhaseField.h, cuPDE.h): the driver's PDE and PhaseField
// (phase_field.h) under the reference's names.
#pragma once
#include "MPIsetting.h"
#include "../phase_field.h"
using cupf_host::PDE;
using cupf_host::PhaseField;
