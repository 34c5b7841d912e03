/* stand-in for OpenGraph's worklist.h (its users are never called here) */
