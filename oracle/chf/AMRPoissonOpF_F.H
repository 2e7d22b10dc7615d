// ORACLE — stands in for the chfpp-generated header of the same name.
#include "chf_oracle.H"
