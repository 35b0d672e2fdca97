/* me_inversion_multi.c -- INVERSION_MULTI (Src/LM_FIT.c:746-811) on the GPU,
 * behind the reference's own signature and structures (see the header). */
#include "me_inversion_multi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static me_plan *g_plan = NULL;
static me_config g_cfg;               /* configuration of g_plan */
static double *g_lambda = NULL;       /* grid of g_plan */
static int g_nl = 0;
static int g_device = 0;
static int g_precision = ME_PREC_FP32;

void me_inversion_multi_set_device(int device) { g_device = device; }
void me_inversion_multi_set_precision(int precision) { g_precision = precision; }

void me_inversion_multi_release(void) {
  if (g_plan) me_plan_destroy(g_plan);
  g_plan = NULL;
  free(g_lambda);
  g_lambda = NULL;
  g_nl = 0;
}

int me_inversion_multi_config(const STRUCT_INPUT *in, const STRUCT_STK *stk,
                              const STRUCT_PARA *para, const STRUCT_LM *lm, me_config *cfg) {
  if (!in || !stk || !para || !lm || !cfg) return ME_ERR_ARG;
  me_config_init(cfg);
  if (para->nline < 1 || para->nline > ME_MAX_LINES || !para->lines || !para->step)
    return ME_ERR_CONFIG;
  /* the line list INIT_INV moved into Para->lines (Src/INV_INIT.c:112-131) */
  cfg->nline = para->nline;
  for (int i = 0; i < para->nline; i++) {
    cfg->line_lambda0[i] = para->lines[i].Lambda0;
    cfg->line_geff[i] = para->lines[i].Geff;
  }
  cfg->lines_seen = 1;
  /* the LM settings INIT_INV copied into STRUCT_LM (Src/INV_INIT.c:187-199) */
  cfg->verbose = lm->verboselv;
  cfg->num_iter = lm->niter;
  cfg->num_run = lm->nruns;
  cfg->convg_criteria = lm->Convg_Criteria;
  cfg->chisq_criteria = lm->Criteria;
  cfg->damp = lm->Damp;
  cfg->lambda_accept = lm->Lam_accept;
  cfg->lambda_reject = lm->Lam_reject;
  cfg->lambda_limits[0] = lm->Lam_Lim[0];
  cfg->lambda_limits[1] = lm->Lam_Lim[1];
  cfg->svd_threshold = lm->Threshold;
  cfg->regul_any = lm->Regul_flag ? 1 : 0;
  cfg->hmi_ref = lm->HMI_REF ? 1 : 0;
  /* the parameter settings in STRUCT_PARA (Src/INV_INIT.c:133-143, 178-179):
   * Limits after INIT_INV's v_los clip, which the plan applies again to the
   * same effect */
  for (int i = 0; i < 9; i++) {
    cfg->bounds[i][0] = para->Limits[i][0];
    cfg->bounds[i][1] = para->Limits[i][1];
    cfg->fixed[i] = para->inv[i] ? 0 : 1;
    cfg->regul[i] = para->regl[i] ? 1 : 0;
    cfg->regul_value[i] = para->value_const[i];
    cfg->regul_weight[i] = para->Regul_weight[i];
    cfg->step[i] = para->step[i];
  }
  cfg->vcoeffi = para->VCoeffi;
  cfg->lcoeffi = para->LCoeffi;
  /* the Stokes settings in STRUCT_STK (Src/INV_INIT.c:201-203, 280-283) */
  for (int s = 0; s < 4; s++) cfg->weights[s] = stk->Weights[s];
  cfg->icriteria = stk->Icriteria;
  cfg->nfigures = stk->Fadd.nfigures;
  /* driver settings left in STRUCT_INPUT */
  cfg->output_fit = in->output_fit ? 1 : 0;
  cfg->cache_prof = in->cache_prof ? 1 : 0;
  cfg->cache_inv = in->cache_inv ? 1 : 0;
  cfg->nprofiles = in->nProf;
  cfg->precision = g_precision;
  return ME_OK;
}

/* The cached plan, remade when the grid or the configuration changed. */
static int plan_for(const STRUCT_INPUT *in, const STRUCT_STK *stk, const STRUCT_PARA *para,
                    const STRUCT_LM *lm, me_plan **out) {
  me_config cfg;
  int st = me_inversion_multi_config(in, stk, para, lm, &cfg);
  if (st != ME_OK) return st;
  const int same = g_plan && g_nl == stk->nw &&
                   memcmp(g_lambda, stk->Lambda, sizeof(double) * (size_t)stk->nw) == 0 &&
                   memcmp(&g_cfg, &cfg, sizeof(cfg)) == 0;
  if (!same) {
    me_inversion_multi_release();
    st = me_plan_create(&cfg, stk->Lambda, stk->nw, g_device, &g_plan);
    if (st != ME_OK) {
      g_plan = NULL;
      return st;
    }
    g_lambda = (double *)malloc(sizeof(double) * (size_t)stk->nw);
    if (!g_lambda) {
      me_inversion_multi_release();
      return ME_ERR_NOMEM;
    }
    memcpy(g_lambda, stk->Lambda, sizeof(double) * (size_t)stk->nw);
    g_nl = stk->nw;
    g_cfg = cfg;
  }
  *out = g_plan;
  return ME_OK;
}

int me_inversion_multi(STRUCT_INPUT *Input, STRUCT_STK *Stk, STRUCT_PARA *Para, STRUCT_LM *LM,
                       STRUCT_SUBSET *Subset) {
  if (!Input || !Stk || !Para || !LM || !Subset) return ME_ERR_ARG;
  me_plan *plan = NULL;
  int st = plan_for(Input, Stk, Para, LM, &plan);
  if (st != ME_OK) {
    fprintf(stderr, "me_inversion_multi: %s (%s)\n", me_strerror(st), me_last_error());
    return st;
  }
  /* LM->chisq carries the last trial's chi^2 from pixel to pixel and from
   * chunk to chunk (Src/LM_FIT.c:555-559) */
  me_plan_set_carry_chisq(plan, LM->chisq);
  st = me_invert_batch(plan, Input->profbuff, Subset->nProf, Input->resbuff,
                       Input->output_fit ? Input->fitbuff : NULL, NULL);
  if (st != ME_OK) {
    fprintf(stderr, "me_inversion_multi: %s (%s)\n", me_strerror(st), me_last_error());
    return st;
  }
  LM->chisq = me_plan_get_carry_chisq(plan);
  return 0;
}
