/*
 * plan.c -- group an ordered list of Pauli rotations into state sweeps
 * ("passes") for the coset kernel in engine.cu.
 *
 * A rotation exp(i phi P) with flip mask f pairs amplitude g with g ^ f.
 * For a run of consecutive rotations whose flip masks lie in a GF(2) space
 * S = span(b_0 .. b_{M-1}), every coset x + S is closed under all of them.
 * The kernel gives each thread whole cosets: it loads the 2^M amplitudes
 * x ^ off(u), off(u) = xor of b_k over the bits k of u, applies the run in
 * registers in the original order, and stores them back.  Per amplitude the
 * arithmetic is exactly the reference's one-rotation-at-a-time update
 * (phase2/qreg_qreg.c:149-160), so grouping never reorders work and the
 * FP64 result is unchanged; only the number of HBM sweeps drops.
 *
 * The planner is greedy and order preserving: it appends rotations to the
 * current pass while the span dimension stays <= max_span (diagonal terms,
 * f = 0, always fit) and starts a new pass otherwise.  Representatives x
 * are the indices with zero bits at the pivots of a reduced echelon form
 * of S; because the basis restricted to the pivot columns is invertible,
 * (x, u) -> x ^ off(u) enumerates every amplitude exactly once.
 *
 * Each rotation is stored in slot coordinates:
 *   U      coefficient vector of f in the basis (partner of slot u is u^U);
 *   odd    (1 - popcount(f & z)) & 1 -- the partner is multiplied by i;
 *   smask  bit u = parity(u & W) ^ (((1 - popcount(f & z)) & 3) >> 1),
 *          W bit k = parity(b_k & z);
 * and the thread adds parity(x & z).  Then slot u is updated as
 *   a_u <- c a_u + (-1)^sigma_u s (odd ? i : 1) a_{u^U},
 * which equals a_g <- c a_g + i s conj(z_g) a_{g^f} with z_g = i^r(g),
 * r(g) = popcount(f & z) + 2 popcount(g & z)  (include/phase2/paulis.h:137-144).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "phase2_b200.h"

#include "p2_internal.h"
#include "plan_core.h"

void p2_sweep_for(uint32_t nqb, int form, int *k, int *low)
{
	int tile = 0, lw = 0;
	p2d_get_sweep(&tile, &lw);
	if (tile > 0 && form == PHASE2_FORM_LIFTED_F32 && nqb <= 31 &&
		nqb >= (uint32_t)tile + 3) {
		*k = tile - lw;
		*low = lw;
	} else {
		*k = 0;
		*low = 0;
	}
}

long phase2_plan(uint32_t nqb, const struct phase2_rot_in *rots, size_t n,
	int max_span, int max_rots, int prec, struct phase2_pass *passes,
	struct phase2_rot_rec *recs)
{
	if (prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32)
		return -1;
	const int form = p2_form_for(prec);
	int k, low;
	p2_sweep_for(nqb, form, &k, &low);
	return p2_plan(nqb, rots, n, max_span, max_rots, P2_DEFAULT_PAD_SPAN,
		form, k, low, passes, recs);
}

long p2_plan(uint32_t nqb, const struct phase2_rot_in *rots, size_t n,
	int max_span, int max_rots, int pad_span, int form, int sweep_k,
	int sweep_low, struct phase2_pass *passes,
	struct phase2_rot_rec *recs)
{
	return p2_plan_core(nqb, rots, NULL, n, max_span, max_rots, pad_span,
		form, sweep_k, sweep_low, passes, recs);
}
