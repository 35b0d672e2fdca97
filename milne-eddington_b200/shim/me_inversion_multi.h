/* me_inversion_multi.h -- the reference-side adapter of libme_b200.
 *
 * A drop-in for the reference's pixel-loop entry point
 *     int INVERSION_MULTI(STRUCT_INPUT *, STRUCT_STK *, STRUCT_PARA *,
 *                         STRUCT_LM *, STRUCT_SUBSET *);       (Src/LM_FIT.h:43-44)
 * with the same signature and the same buffers: Subset->nProf pixels of
 * Input->profbuff [nProf][4][Stk->nw] in, Input->resbuff [nProf][10] (and, with
 * Input->output_fit, Input->fitbuff) out, zeros for skipped pixels, the LM
 * chi^2 carried from pixel to pixel in LM->chisq.  It is compiled against the
 * reference's own headers (RINPUT.h, ME_SOLVER.h, LM_FIT.h) and linked with
 * libme_b200.so, so the reference's driver (Src/ME_INV.c:115, 128, 271) calls
 * it unchanged after
 *     #define INVERSION_MULTI me_inversion_multi
 * The configuration comes from the structures RDINPUT and INIT_INV filled;
 * the plan (device buffers, constants) is made on the first call and reused
 * while the grid and the configuration stay the same.
 */
#ifndef ME_INVERSION_MULTI_H
#define ME_INVERSION_MULTI_H

#include "RINPUT.h"
#include "ME_SOLVER.h"
#include "LM_FIT.h"
#include "me_b200.h"

/* INVERSION_MULTI on the GPU.  Returns 0, or a negative ME_* status (where the
 * reference would have stopped the program); me_last_error() says why. */
int me_inversion_multi(STRUCT_INPUT *Input, STRUCT_STK *Stk, STRUCT_PARA *Para, STRUCT_LM *LM,
                       STRUCT_SUBSET *Subset);

/* The me_config of the settings INVERSION_MULTI reads, from the structures as
 * RDINPUT and INIT_INV left them (the line list in Para->lines, the LM settings
 * in LM, the Stokes weights and Icriteria in Stk; theta / phi limits and
 * regularisation values in radians). */
int me_inversion_multi_config(const STRUCT_INPUT *Input, const STRUCT_STK *Stk,
                              const STRUCT_PARA *Para, const STRUCT_LM *LM, me_config *cfg);

/* The CUDA device (default 0) and synthesis precision (ME_PREC_FP32, the
 * default, or ME_PREC_FP64) of the plans made from now on. */
void me_inversion_multi_set_device(int device);
void me_inversion_multi_set_precision(int precision);

/* Destroys the cached plan (at the end of the program). */
void me_inversion_multi_release(void);

#endif
