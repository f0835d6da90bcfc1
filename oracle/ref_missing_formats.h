// ref_missing_formats.h -- TEST INFRASTRUCTURE ONLY.
//
// The reference's blockwise_individual.h:66-68,119-120,212-213 and
// exhaustive_size_format_selector.h:127,129 name two default cascades that no
// header of the reference defines, so neither compiles as shipped.  They are
// the delta and FOR cascades over the default group_simple format, written
// here the way default_formats.h:54-82 writes the same cascades over
// dynamic_vbp.  Included (with -include) before the reference's headers by
// oracle/Makefile for ref_bwi.cpp only.
#ifndef MS_ORACLE_REF_MISSING_FORMATS_H
#define MS_ORACLE_REF_MISSING_FORMATS_H

#include <core/morphing/default_formats.h>

#define DEFAULT_DELTA_GROUP_SIMPLE_F(ve) \
    SINGLE_ARG(delta_f<1024, ve::vector_helper_t::element_count::value, DEFAULT_GROUP_SIMPLE_F(ve)>)

#define DEFAULT_FOR_GROUP_SIMPLE_F(ve) \
    SINGLE_ARG(for_f<1024, ve::vector_helper_t::element_count::value, DEFAULT_GROUP_SIMPLE_F(ve)>)

#endif
