/* Abort-stubs for the 34 Fortran REFPROP entry points of the reference's
 * NISTThermo package (test infrastructure only).  MPFLOW3D's EOS layer links
 * them for MATERIAL_TYPE_NIST (EOS/src/EOS_NIST.c); with
 * MATERIAL_TYPE_IDEALGAS, the only material the oracle runs, none of them is
 * ever called (EOS/src/EOS.c:22-40,196-215), and there is no Fortran compiler
 * here to build them.  Calling one aborts the oracle process loudly. */
#include <stdio.h>
#include <stdlib.h>

#define NIST_STUB(name)                                                              \
    void name(void) {                                                                \
        fprintf(stderr, "oracle: NIST routine " #name " called on the ideal-gas path\n"); \
        abort();                                                                     \
    }

NIST_STUB(critp_) NIST_STUB(dhd1_) NIST_STUB(dhflsh_) NIST_STUB(dpdd2_) NIST_STUB(dpdd_) NIST_STUB(dpdt_)
NIST_STUB(fgcty_) NIST_STUB(info_) NIST_STUB(limitk_) NIST_STUB(meltp_) NIST_STUB(meltt_)
NIST_STUB(pdepdflsh2_) NIST_STUB(pdepdflsh_) NIST_STUB(pdflsh_) NIST_STUB(phflsh_) NIST_STUB(press_)
NIST_STUB(psflsh_) NIST_STUB(satp_) NIST_STUB(satt_) NIST_STUB(setpath_) NIST_STUB(setup_) NIST_STUB(sublp_)
NIST_STUB(sublt_) NIST_STUB(surft_) NIST_STUB(tdetdflsh2_) NIST_STUB(tdetdflsh_) NIST_STUB(tdflsh_)
NIST_STUB(therm_) NIST_STUB(thflsh_) NIST_STUB(tpflsh_) NIST_STUB(tprho_) NIST_STUB(trnprp_) NIST_STUB(virb_)
NIST_STUB(virc_)
