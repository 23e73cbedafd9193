<?xml version="1.0"?>
<!-- nb_dof 2, negative and multi-digit marks, sides with negative marks -->
<OFELI_File>
<info><title>codes</title></info>
<Mesh nb_dof="2"   dim="2" >
   <Nodes>
	0.0 0.0 11
   1.0  0.0   -12
   1.0 1.0 3
 0.0 1.0 -1
 0.5 0.5 0
 1e-1 2.5E-1 120
 0.3333333333333333 -7.25e-3 -99
   </Nodes>
   <!-- four triangles around the centre -->
   <Elements shape="tria" nodes="3">
 1 2 5 3
 2 3 5 3
 3 4 5 3
 4 1 5 3
   </Elements>
   <Sides nodes="2"shape="line">
 1 2 -21
 2 3 10
 3 4 0
 4 1 -3
   </Sides>
</Mesh>
</OFELI_File>
