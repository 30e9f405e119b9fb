// Src/Hierarchy.h of the drop-in layer: the reference's header of this name
// (found next on the include path), then the device forwarding of its solve
// path (gdtp_dropin.inl).  Put this repository's include/ directory before the
// reference's.
#pragma once
#include_next <Src/Hierarchy.h>
#include "gdtp_dropin.inl"
