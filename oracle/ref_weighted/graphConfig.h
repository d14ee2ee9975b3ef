/* Shadow of 00_graph_bench/include/config/graphConfig.h for the WEIGHTED=1
 * build of the reference (oracle/_ref/libogref_w.so).  The reference header
 * hard-codes WEIGHTED 0; this file is found first on the include path and
 * differs only in that macro.  struct Arguments must stay byte-identical to
 * the reference's (graphConfig.h:11-44). */
#ifndef GRAPHCONFIG_H
#define GRAPHCONFIG_H

#include <stdint.h>
#include "mt19937.h"

#define WEIGHTED 1
#define DIRECTED 1

struct Arguments
{
    int wflag;
    int xflag;
    int sflag;
    int Sflag;
    int dflag;
    uint32_t binSize;
    uint32_t verbosity;
    uint32_t iterations;
    uint32_t trials;
    double epsilon;
    int source;
    uint32_t algorithm;
    uint32_t datastructure;
    uint32_t pushpull;
    uint32_t sort;
    uint32_t lmode;
    uint32_t lmode_l2;
    uint32_t lmode_l3;
    uint32_t mmode;
    uint32_t symmetric;
    uint32_t weighted;
    uint32_t delta;
    int pre_numThreads;
    int algo_numThreads;
    int ker_numThreads;
    char *fnameb;
    char *fnamel;
    uint32_t fnameb_format;
    uint32_t convert_format;
    mt19937state mt19937var;
    uint32_t cache_size;
};

#endif
