/* stand-in for OpenGraph's fixedPoint.h (its users are never called here) */
