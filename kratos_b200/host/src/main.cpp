// Entry point (src/main.cpp of the reference): prob::run with the parameter files.
#include <iostream>
#include <stdexcept>
#include "user/probgen.h"

int main( int argc, char * argv[  ] )
{
    if( argc <= 1 )
        throw std::runtime_error( "No input file." );
    prob::run( argc, argv );
    return 0;
}
