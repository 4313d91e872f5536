/* Empty: the reference includes this header (patchtable.h:8) but uses none of it on the oracle path. */
