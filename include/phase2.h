#ifndef PHASE2_H
#define PHASE2_H

/* Umbrella header, as include/phase2.h of Quantum-for-Life/phase2. */

#include <stddef.h>

#include "phase2/circ.h"
#include "phase2/paulis.h"
#include "phase2/qreg.h"
#include "phase2/step_writer.h"
#include "phase2/world.h"
#include "prob.h"

#endif /* PHASE2_H */
