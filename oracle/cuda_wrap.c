/*
 * cuda_wrap.c -- TEST INFRASTRUCTURE: lets the reference's own qLD-compute
 * binary run the -cuda compute without touching its sources.
 *
 * oracle/Makefile links the unmodified correlator objects with
 * -Wl,--wrap=correlate, so every call correlate_function() makes to
 * correlate() (src/correlator/src/correlate_function.c:242-256,268-282)
 * lands here.  With QLD_CUDA set in the environment the call goes to
 * correlate_cuda() (qld_b200/host/correlate_cuda.c, same arguments);
 * otherwise to the reference's correlate().  The real integration adds a
 * -cuda flag to qLD-compute instead, which selects correlate_cuda() in the
 * same place.
 */
#include <stdlib.h>

#include "gemm_cpu.h"

void __real_correlate(threadData_t *threadData, outFileType fpOut,
                      inputDataType_x64 *tableA, unsigned int *tableA_posIndex,
                      char **tableA_IDindex, unsigned int *tableA_bitcount, int tableAsize,
                      inputDataType_x64 *tableB, unsigned int *tableB_posIndex,
                      char **tableB_IDindex, unsigned int *tableB_bitcount, int tableBsize,
                      int compressed_snp_size, int snp_size, int posWset2);

void correlate_cuda(threadData_t *threadData, outFileType fpOut,
                    inputDataType_x64 *tableA, unsigned int *tableA_posIndex,
                    char **tableA_IDindex, unsigned int *tableA_bitcount, int tableAsize,
                    inputDataType_x64 *tableB, unsigned int *tableB_posIndex,
                    char **tableB_IDindex, unsigned int *tableB_bitcount, int tableBsize,
                    int compressed_snp_size, int snp_size, int posWset2);

void __wrap_correlate(threadData_t *threadData, outFileType fpOut,
                      inputDataType_x64 *tableA, unsigned int *tableA_posIndex,
                      char **tableA_IDindex, unsigned int *tableA_bitcount, int tableAsize,
                      inputDataType_x64 *tableB, unsigned int *tableB_posIndex,
                      char **tableB_IDindex, unsigned int *tableB_bitcount, int tableBsize,
                      int compressed_snp_size, int snp_size, int posWset2)
{
    if (getenv("QLD_CUDA"))
        correlate_cuda(threadData, fpOut, tableA, tableA_posIndex, tableA_IDindex,
                       tableA_bitcount, tableAsize, tableB, tableB_posIndex, tableB_IDindex,
                       tableB_bitcount, tableBsize, compressed_snp_size, snp_size, posWset2);
    else
        __real_correlate(threadData, fpOut, tableA, tableA_posIndex, tableA_IDindex,
                         tableA_bitcount, tableAsize, tableB, tableB_posIndex, tableB_IDindex,
                         tableB_bitcount, tableBsize, compressed_snp_size, snp_size, posWset2);
}
