<?xml version='1.0'?>
<case codeversion="1.0" codename="Mahyco" xml:lang="en">
  <arcane>
    <title>bisod_remap_superbee</title>
    <timeloop>MahycoLoop</timeloop>
  </arcane>
  <mesh>
    <meshgenerator>
      <cartesian>
        <nsd>1 1 1</nsd>
        <origine>0.0 0.0 0.0</origine>
        <lx nx='64' prx='1.0'>1.</lx>
        <ly ny='8' pry='1.0'>0.25</ly>
        <lz nz='8' prz='1.0'>0.25</lz>
      </cartesian>
    </meshgenerator>
  </mesh>
  <time-history>
    <bilan name="EnvSummation">
      <periode>5</periode>
      <variable>Density</variable>
    </bilan>
  </time-history>
  <mahyco>
    <material><name>L_mat</name></material>
    <material><name>R_mat</name></material>
    <environment>
      <name>LEFT</name>
      <material>L_mat</material>
      <densite-initiale>1.</densite-initiale>
      <pression-initiale>1.</pression-initiale>
      <eos-model name="PerfectGas">
        <adiabatic-cst>1.4</adiabatic-cst>
      </eos-model>
    </environment>
    <environment>
      <name>RIGHT</name>
      <material>R_mat</material>
      <densite-initiale>0.125</densite-initiale>
      <pression-initiale>0.1</pression-initiale>
      <eos-model name="StiffenedGas">
        <adiabatic-cst>1.4</adiabatic-cst>
        <limit-tension>0.02</limit-tension>
      </eos-model>
    </environment>
    <cas-model name="SOD">
      <cas-test>13</cas-test>
    </cas-model>
    <remap name="RemapADI">
      <ordre-projection>2</ordre-projection>
      <projection-limiteur-id>1</projection-limiteur-id>
    </remap>
    <pseudo-centree>0</pseudo-centree>
    <schema-csts>0</schema-csts>
    <cfl>0.25</cfl>
    <deltat-init>0.00001</deltat-init>
    <deltat-min>0.00000001</deltat-min>
    <deltat-max>0.01</deltat-max>
    <longueur-caracteristique>racine-cubique-volume</longueur-caracteristique>
    <final-time>.2</final-time>
    <boundary-condition><surface>XMIN</surface><type>Vx</type><value>0.</value></boundary-condition>
    <boundary-condition><surface>XMAX</surface><type>Vx</type><value>0.</value></boundary-condition>
    <boundary-condition><surface>YMIN</surface><type>Vy</type><value>0.</value></boundary-condition>
    <boundary-condition><surface>YMAX</surface><type>Vy</type><value>0.</value></boundary-condition>
    <boundary-condition><surface>ZMIN</surface><type>Vz</type><value>0.</value></boundary-condition>
    <boundary-condition><surface>ZMAX</surface><type>Vz</type><value>0.</value></boundary-condition>
  </mahyco>
</case>
