/* The device table of TBTK's GPUResourceManager over libtbtkkpm.
 *
 * Drop-in for Lib/src/cuda/GPUResourceManager.cu and
 * Lib/src/nocuda/GPUResourceManager.cpp, the two files TBTK chooses between
 * to provide GPUResourceManager::createDeviceTable / destroyDeviceTable
 * (Lib/include/Utilities/TBTK/GPUResourceManager.h:62-66).  The device count
 * comes from tbtkkpm_device_count, so the pool that allocateDevice /
 * freeDevice hand out (Lib/src/Utilities/GPUResourceManager.cpp:44-90) is the
 * set of devices the B200 library can use.
 */
#include "TBTK/GPUResourceManager.h"
#include "TBTK/Streams.h"

#include "tbtkkpm.h"

namespace TBTK{

void GPUResourceManager::createDeviceTable(){
	int count = 0;
	if(tbtkkpm_device_count(&count) != TBTKKPM_OK)
		count = 0;
	numDevices = count;

	if(getGlobalVerbose())
		Streams::out << "Num GPU devices: " << numDevices << "\n";

	if(numDevices > 0){
		busyDevices = new bool[numDevices];
		for(int n = 0; n < numDevices; n++)
			busyDevices[n] = false;
	}
}

void GPUResourceManager::destroyDeviceTable(){
	if(numDevices > 0){
		delete [] busyDevices;
		busyDevices = nullptr;
	}
}

};	//End of namespace TBTK
