// Test infrastructure: empty stand-in for a SCUFF-EM interpolation header that
// the reference's GetFields.cc includes without using on the field path.
