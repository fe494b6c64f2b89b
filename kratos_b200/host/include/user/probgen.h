// Problem-generator entry (src/user/probgen.h of the reference): main calls
// prob::run; prob::cmd reads every parameter file named on the command line,
// later ones overriding earlier ones.
#pragma once

#include "../io/args/input.h"

namespace prob
{
void cmd( int argc, char * argv[  ], input & args );
void run( int argc, char * argv[  ] );
}
