/*
 * TEST INFRASTRUCTURE (oracle).  Plain-C rank-d complex DFT (see oracle_dft.c).
 */
#ifndef ORACLE_DFT_H
#define ORACLE_DFT_H
#ifdef __cplusplus
extern "C" {
#endif
/* In-place unnormalised DFT of a row-major complex array of shape dims[rank].
 * Element e (row-major index) lives at data[2*e*stride], data[2*e*stride+1].
 * sign = -1 (FFTW_FORWARD) or +1 (FFTW_BACKWARD). */
void oracle_dft_nd(double *data, int rank, const int *dims, long stride,
                   int sign);
#ifdef __cplusplus
}
#endif
#endif
