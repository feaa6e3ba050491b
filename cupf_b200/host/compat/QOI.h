// QOI.h — for callers written against the reference's headers (3DgrainMPI/QOI.h):
// the driver's QoI classes (qoi.h) under the reference's names.
#pragma once
#include "MPIsetting.h"
#include "../phase_field.h"
using cupf_host::QOI;
using cupf_host::QOI3D;
using cupf_host::QOILine;
