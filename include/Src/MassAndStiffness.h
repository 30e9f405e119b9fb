// Src/MassAndStiffness.h of the drop-in layer: the reference's header of this
// name (found next on the include path), the forwarding of Src/Hierarchy.h, and
// the recording wrapper of InitializeMassAndStiffness (gdtp_dropin_assembly.inl).
#pragma once
#include_next <Src/MassAndStiffness.h>
#include <Src/Hierarchy.h>
#include "gdtp_dropin_assembly.inl"
