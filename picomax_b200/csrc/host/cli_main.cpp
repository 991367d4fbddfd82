// The picomax executable: argv in, .dat/.gpt out (reference: src/pmx.cpp:43).
#include "../../../include/picomax.h"

int main(int argc, char** argv) { return pmx_main(argc, const_cast<const char* const*>(argv)); }
