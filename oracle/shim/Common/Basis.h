// kmc/Event.h includes "../Common/Basis.h" relative to its own directory, where the
// reference tree has no Basis.h; with -Ishim/Common this path resolves here and forwards to
// the project's stand-in, with the species table (potentials/Species.h) the reference's
// Basis.h brings along for Event::writeSaddle.  Test infrastructure only.
#pragma once
#include "Species.h"
#include "../Basis.h"
