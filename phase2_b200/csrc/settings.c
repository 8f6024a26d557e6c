/*
 * settings.c -- process-wide defaults of the B200 extensions
 * (include/phase2_b200.h): precision, fusion policy and term order.
 */
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "cfg"
#include "log.h"

#include "phase2_b200.h"

#include "p2_host.h"

struct p2_settings p2_cfg = {
	.prec = PHASE2_PREC_FP64,
	.max_span = PHASE2_MAX_SPAN,
	.max_rots = 0,
	.order = PHASE2_ORDER_LEX,
	.fp32_form = PHASE2_FORM_LIFTED_MIXED,
	.batch_persistent = 1,
	.device_sampling = PHASE2_DEVICE_SAMPLING_AUTO,
};

void p2_settings_from_env(void)
{
	const char *p = getenv("PHASE2_PRECISION");
	if (p && *p) {
		if (!strcmp(p, "fp32") || !strcmp(p, "FP32"))
			p2_cfg.prec = PHASE2_PREC_FP32;
		else if (!strcmp(p, "fp64") || !strcmp(p, "FP64"))
			p2_cfg.prec = PHASE2_PREC_FP64;
		else
			log_warn("PHASE2_PRECISION=%s not understood", p);
	}
	const char *f = getenv("PHASE2_FP32_FORM");
	if (f && *f) {
		if (!strcmp(f, "lifted"))
			p2_cfg.fp32_form = PHASE2_FORM_LIFTED;
		else if (!strcmp(f, "lifted_f32"))
			p2_cfg.fp32_form = PHASE2_FORM_LIFTED_F32;
		else if (!strcmp(f, "mixed"))
			p2_cfg.fp32_form = PHASE2_FORM_LIFTED_MIXED;
		else
			log_warn("PHASE2_FP32_FORM=%s not understood", f);
	}
	const char *d = getenv("PHASE2_DEVICE_SAMPLING");
	if (d && *d) {
		if (!strcmp(d, "0") || !strcmp(d, "off"))
			p2_cfg.device_sampling = PHASE2_DEVICE_SAMPLING_OFF;
		else if (!strcmp(d, "1") || !strcmp(d, "on"))
			p2_cfg.device_sampling = PHASE2_DEVICE_SAMPLING_ON;
		else if (!strcmp(d, "auto"))
			p2_cfg.device_sampling = PHASE2_DEVICE_SAMPLING_AUTO;
		else
			log_warn("PHASE2_DEVICE_SAMPLING=%s not understood", d);
	}
}

int phase2_set_fp32_form(int form)
{
	if (form != PHASE2_FORM_LIFTED && form != PHASE2_FORM_LIFTED_F32 &&
		form != PHASE2_FORM_LIFTED_MIXED)
		return -1;
	p2_cfg.fp32_form = form;
	return 0;
}

int phase2_get_fp32_form(void)
{
	return p2_cfg.fp32_form;
}

int phase2_set_batch_persistent(int on)
{
	p2_cfg.batch_persistent = on ? 1 : 0;
	return 0;
}

int phase2_set_sweep(int tile_qubits, int low_qubits)
{
	return p2d_set_sweep(tile_qubits, low_qubits);
}

void phase2_get_sweep(int *tile_qubits, int *low_qubits)
{
	p2d_get_sweep(tile_qubits, low_qubits);
}

int phase2_set_sweep_kernel(int on)
{
	p2d_set_sweep_kernel(on);
	return 0;
}

int phase2_set_device_sampling(int mode)
{
	if (mode != PHASE2_DEVICE_SAMPLING_OFF &&
		mode != PHASE2_DEVICE_SAMPLING_ON &&
		mode != PHASE2_DEVICE_SAMPLING_AUTO)
		return -1;
	p2_cfg.device_sampling = mode;
	return 0;
}

int p2_form_for(int prec)
{
	return prec == PHASE2_PREC_FP32 ? p2_cfg.fp32_form : PHASE2_FORM_EXACT;
}

int phase2_set_precision(int prec)
{
	if (prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32)
		return -1;
	p2_cfg.prec = prec;
	return 0;
}

int phase2_get_precision(void)
{
	return p2_cfg.prec;
}

int phase2_set_fusion(int max_span, int max_rots)
{
	if (max_span < 1 || max_span > PHASE2_MAX_SPAN || max_rots < 0)
		return -1;
	p2_cfg.max_span = max_span;
	p2_cfg.max_rots = max_rots;
	return 0;
}

int phase2_set_term_order(int order)
{
	if (order != PHASE2_ORDER_LEX && order != PHASE2_ORDER_GIVEN &&
		order != PHASE2_ORDER_FLIP)
		return -1;
	p2_cfg.order = order;
	return 0;
}

int phase2_get_term_order(void)
{
	return p2_cfg.order;
}

const char *phase2_version(void)
{
	return "phase2-b200 0.1.0 (sm_100a)";
}
