/* Test infrastructure: CPU DFT restatement (see dft.c). */
#ifndef ORACLE_DFT_H
#define ORACLE_DFT_H

void oracle_dft_1d(double *data, int n, long stride, int sign);
void oracle_dft_nd(double *data, int rank, const int *dims, int sign);
void oracle_dft_r2c_3d(const double *in, long in_row, double *out, long out_row, int n0, int n1, int n2);
void oracle_dft_c2r_3d(const double *in, long in_row, double *out, long out_row, int n0, int n1, int n2);

#endif
