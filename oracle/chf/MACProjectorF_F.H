// ORACLE — stands in for the chfpp-generated header of the same name;
// no kernel of it is called on the solve path.
