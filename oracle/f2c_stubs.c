/* Link-time stand-ins for the f2c runtime routines referenced by the reference's GENESIS (FEL)
 * sources. The reference's srwlib.cpp links GENESIS in, but the propagation path never calls it;
 * each stand-in aborts if it is ever reached, so a stray call cannot go unnoticed.
 * Test infrastructure only (part of the oracle build recipe). */
#include <stdio.h>
#include <stdlib.h>
#define F2C_STUB(name) int name() { fprintf(stderr, "f2c routine " #name " called (not built)\n"); abort(); return 0; }
F2C_STUB(d_cnjg) F2C_STUB(d_imag) F2C_STUB(d_mod) F2C_STUB(d_sign) F2C_STUB(do_fio) F2C_STUB(do_lio)
F2C_STUB(do_uio) F2C_STUB(e_rdue) F2C_STUB(e_rsfe) F2C_STUB(e_rsli) F2C_STUB(e_wdue) F2C_STUB(e_wsfe)
F2C_STUB(e_wsfi) F2C_STUB(e_wsle) F2C_STUB(e_wsli) F2C_STUB(f_clos) F2C_STUB(f_inqu) F2C_STUB(f_open)
F2C_STUB(f_rew) F2C_STUB(i_dnnt) F2C_STUB(i_indx) F2C_STUB(i_len) F2C_STUB(pow_ii) F2C_STUB(pow_ri)
F2C_STUB(s_cat) F2C_STUB(s_cmp) F2C_STUB(s_copy) F2C_STUB(s_rdue) F2C_STUB(s_rsfe) F2C_STUB(s_rsli)
F2C_STUB(s_stop) F2C_STUB(s_wdue) F2C_STUB(s_wsfe) F2C_STUB(s_wsfi) F2C_STUB(s_wsle) F2C_STUB(s_wsli)
F2C_STUB(z_div) F2C_STUB(z_exp)
