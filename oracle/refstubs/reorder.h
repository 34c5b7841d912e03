/* stand-in for OpenGraph's reorder.h (its users are never called here) */
