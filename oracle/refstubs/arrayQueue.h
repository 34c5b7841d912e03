/* stand-in for OpenGraph's arrayQueue.h (its users are never called here) */
