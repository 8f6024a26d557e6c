/*
 * layout.c -- sizeof table for FFI bindings (phase2_sizeof).
 */
#include "circ/cmpsit.h"
#include "circ/qdrift.h"
#include "circ/trott.h"
#include "circ/trott2.h"
#include "phase2_b200.h"

size_t phase2_sizeof(int which)
{
	switch (which) {
	case 0:
		return sizeof(struct qreg);
	case 1:
		return sizeof(struct circ);
	case 2:
		return sizeof(struct trott);
	case 3:
		return sizeof(struct trott2);
	case 4:
		return sizeof(struct qdrift);
	case 5:
		return sizeof(struct cmpsit);
	case 6:
		return sizeof(struct circ_hamil_term);
	case 7:
		return sizeof(struct phase2_pass);
	case 8:
		return sizeof(struct phase2_rot_rec);
	case 9:
		return sizeof(struct phase2_stats);
	default:
		return 0;
	}
}
