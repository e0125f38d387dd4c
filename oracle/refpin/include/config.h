/* Test infrastructure: the reference's autoconf header is generated by its
   build system, which the pin does not run; OpenMP is switched on from the
   compiler command line instead. */
