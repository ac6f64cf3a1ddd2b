// Stand-in for the alien/AlienConfig.h that Alien's CMake configure step
// generates from src/AlienConfig.h.in (TEST INFRASTRUCTURE): the macros the
// back-end headers use.
#pragma once
#define ALIEN_UNUSED(var) \
  do {                    \
    (void)(var);          \
  } while (0)
#ifndef ALIEN_UNUSED_PARAM
#define ALIEN_UNUSED_PARAM [[maybe_unused]]
#endif
