// Stand-in for the generated alien/AlienExport.h (TEST INFRASTRUCTURE): a
// static, single-library test build needs no symbol-visibility attributes.
#pragma once
#define ALIEN_EXPORT
