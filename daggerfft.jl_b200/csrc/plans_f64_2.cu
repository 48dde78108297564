// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<double,true,1024,3,1,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,3,1,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,10,1,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,10,1,10>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,10,1,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,10,1,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,24,4,6,4>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,24,4,6,4>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,24,4,6,4>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,24,4,6,4>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,40,5,5,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,40,5,5,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,40,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,40,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,64,8,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,64,8,8,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,64,8,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,64,8,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,96,8,12,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,96,8,12,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,96,8,12,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,96,8,12,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,135,9,15,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,135,9,15,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,135,9,15,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,135,9,15,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,192,12,12,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,192,12,12,16>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,192,12,12,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,192,12,12,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,250,25,10,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,250,25,10,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,250,25,10,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,250,25,10,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,324,54,6,6,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,324,54,6,6,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,324,54,6,6,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,324,54,6,6,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,432,36,12,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,432,36,12,6,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,432,36,12,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,432,36,12,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,540,36,15,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,540,36,15,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,675,45,15,15,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,675,45,15,15,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,810,54,15,6,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,810,54,15,6,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1024,64,16,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1024,64,16,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1250,125,10,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1250,125,10,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1500,100,15,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1500,100,15,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1875,125,15,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1875,125,15,5,5,5>(const PassDesc);
extern const StaticPlan kPlans_f64_2[];
extern const int kPlansCount_f64_2;
const StaticPlan kPlans_f64_2[] = {
  {3, 1, 1, {3}, 1024, (const void*)&axis_pass_static<double,true,1024,3,1,3>, (const void*)&axis_pass_static<double,false,1024,3,1,3>, nullptr, nullptr, 512, 0},
  {10, 1, 1, {10}, 512, (const void*)&axis_pass_static<double,true,512,10,1,10>, (const void*)&axis_pass_static<double,false,512,10,1,10>, (const void*)&axis_pass_pipe<double,512,false,8,10,1,10>, (const void*)&axis_pass_pipe<double,512,true,0,10,1,10>, 512, 8},
  {24, 4, 2, {6,4}, 1024, (const void*)&axis_pass_static<double,true,1024,24,4,6,4>, (const void*)&axis_pass_static<double,false,1024,24,4,6,4>, (const void*)&axis_pass_pipe<double,512,false,8,24,4,6,4>, (const void*)&axis_pass_pipe<double,512,true,0,24,4,6,4>, 512, 8},
  {40, 5, 2, {5,8}, 512, (const void*)&axis_pass_static<double,true,512,40,5,5,8>, (const void*)&axis_pass_static<double,false,512,40,5,5,8>, (const void*)&axis_pass_pipe<double,512,false,8,40,5,5,8>, (const void*)&axis_pass_pipe<double,512,true,0,40,5,5,8>, 512, 8},
  {64, 8, 2, {8,8}, 1024, (const void*)&axis_pass_static<double,true,1024,64,8,8,8>, (const void*)&axis_pass_static<double,false,1024,64,8,8,8>, (const void*)&axis_pass_pipe<double,512,false,8,64,8,8,8>, (const void*)&axis_pass_pipe<double,512,true,0,64,8,8,8>, 512, 8},
  {96, 8, 2, {12,8}, 512, (const void*)&axis_pass_static<double,true,512,96,8,12,8>, (const void*)&axis_pass_static<double,false,512,96,8,12,8>, (const void*)&axis_pass_pipe<double,512,false,8,96,8,12,8>, (const void*)&axis_pass_pipe<double,512,true,0,96,8,12,8>, 512, 8},
  {135, 9, 3, {15,3,3}, 512, (const void*)&axis_pass_static<double,true,512,135,9,15,3,3>, (const void*)&axis_pass_static<double,false,512,135,9,15,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,135,9,15,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,135,9,15,3,3>, 512, 8},
  {192, 12, 2, {12,16}, 512, (const void*)&axis_pass_static<double,true,512,192,12,12,16>, (const void*)&axis_pass_static<double,false,512,192,12,12,16>, (const void*)&axis_pass_pipe<double,512,false,8,192,12,12,16>, (const void*)&axis_pass_pipe<double,512,true,0,192,12,12,16>, 512, 8},
  {250, 25, 3, {10,5,5}, 512, (const void*)&axis_pass_static<double,true,512,250,25,10,5,5>, (const void*)&axis_pass_static<double,false,512,250,25,10,5,5>, (const void*)&axis_pass_pipe<double,512,false,8,250,25,10,5,5>, (const void*)&axis_pass_pipe<double,512,true,0,250,25,10,5,5>, 512, 8},
  {324, 54, 4, {6,6,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,324,54,6,6,3,3>, (const void*)&axis_pass_static<double,false,1024,324,54,6,6,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,324,54,6,6,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,324,54,6,6,3,3>, 512, 8},
  {432, 36, 3, {12,6,6}, 512, (const void*)&axis_pass_static<double,true,512,432,36,12,6,6>, (const void*)&axis_pass_static<double,false,512,432,36,12,6,6>, (const void*)&axis_pass_pipe<double,512,false,8,432,36,12,6,6>, (const void*)&axis_pass_pipe<double,512,true,0,432,36,12,6,6>, 512, 8},
  {540, 36, 3, {15,6,6}, 512, (const void*)&axis_pass_static<double,true,512,540,36,15,6,6>, (const void*)&axis_pass_static<double,false,512,540,36,15,6,6>, nullptr, nullptr, 512, 0},
  {675, 45, 3, {15,15,3}, 512, (const void*)&axis_pass_static<double,true,512,675,45,15,15,3>, (const void*)&axis_pass_static<double,false,512,675,45,15,15,3>, nullptr, nullptr, 512, 0},
  {810, 54, 4, {15,6,3,3}, 512, (const void*)&axis_pass_static<double,true,512,810,54,15,6,3,3>, (const void*)&axis_pass_static<double,false,512,810,54,15,6,3,3>, nullptr, nullptr, 512, 0},
  {1024, 64, 3, {16,8,8}, 512, (const void*)&axis_pass_static<double,true,512,1024,64,16,8,8>, (const void*)&axis_pass_static<double,false,512,1024,64,16,8,8>, nullptr, nullptr, 512, 0},
  {1250, 125, 4, {10,5,5,5}, 512, (const void*)&axis_pass_static<double,true,512,1250,125,10,5,5,5>, (const void*)&axis_pass_static<double,false,512,1250,125,10,5,5,5>, nullptr, nullptr, 512, 0},
  {1500, 100, 3, {15,10,10}, 512, (const void*)&axis_pass_static<double,true,512,1500,100,15,10,10>, (const void*)&axis_pass_static<double,false,512,1500,100,15,10,10>, nullptr, nullptr, 512, 0},
  {1875, 125, 4, {15,5,5,5}, 512, (const void*)&axis_pass_static<double,true,512,1875,125,15,5,5,5>, (const void*)&axis_pass_static<double,false,512,1875,125,15,5,5,5>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f64_2 = 18;
}  // namespace dfft
