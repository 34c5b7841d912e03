/* stand-in for OpenGraph's bitmap.h (its users are never called here) */
