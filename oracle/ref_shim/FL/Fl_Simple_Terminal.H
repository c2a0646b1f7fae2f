/* Build shim for compiling FlowLB's solver sources without the FLTK GUI
 * library: the solver path only passes this type around by pointer. */
#pragma once
class Fl_Simple_Terminal;
