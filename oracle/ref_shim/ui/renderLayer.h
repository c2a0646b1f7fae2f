/* Build shim: FlowLB's src/cuda/cudaIsosurface.cuh includes the UI render
 * layer (ImGui, windowing) but its iso-line kernel uses nothing from it. */
#pragma once
