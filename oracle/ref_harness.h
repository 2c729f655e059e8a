/*
 * ref_harness.h - shared handle of the oracle harness.
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is the reference renderer itself,
 * compiled from its own sources by oracle/Makefile into oracle/_ref/. These
 * harness translation units expose the reference's functions (including a
 * few file-static helpers, reached by #including the reference .c file as
 * tests/test_water_units.c:50 does) through a flat C ABI so the tests and the
 * CPU-baseline leg of bench.py can drive them with ctypes. Nothing in the
 * GPU product path links or calls this code.
 */
#ifndef MT_REF_HARNESS_H
#define MT_REF_HARNESS_H

#include "scene.h"
#include "camera.h"

typedef struct {
    Scene  scene;
    Camera cam;
} MtRefHandle;

#endif
